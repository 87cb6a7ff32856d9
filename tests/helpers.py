"""Shared helpers of the tests: run a case through the CUDA path and through a CPU oracle."""
import numpy as np

import compas_b200 as cb
from oracle.oracle import Oracle, have_ref


def oracle_kind(physics, dim, nphase=2):
    return "reference" if have_ref(physics, dim, nphase) else "port"


def rel_linf(a, b):
    """max |a - b| / max |b| per component (the parity norm of the north star)."""
    out = []
    for c in range(a.shape[0]):
        den = float(np.max(np.abs(b[c])))
        out.append(float(np.max(np.abs(a[c] - b[c]))) / (den if den > 0 else 1.0))
    return np.array(out)


def build_case(case_fn, **kw):
    phys, dim, inputs, geom, U = case_fn(**kw)
    p = cb.make_parm(phys, dim, inputs)  # FIVEEQS_NPHASE: nphase from the per-phase lists
    g = cb.make_geom(**geom)
    return p, g, U


def run_gpu(p, g, U, nsteps, use_graph=True, stop_time=1e300):
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(nsteps, stop_time=stop_time, use_graph=use_graph)
    info = lv.sync()
    out = lv.download()
    dts = lv.dts(info.steps)
    lv.close()
    return out, info, dts


def run_oracle(p, g, U, nsteps, kind=None, stop_time=1e300):
    ref = U.copy()
    o = Oracle(kind or oracle_kind(p.physics, p.dim, p.nphase), p, g)
    t, dts = o.advance(ref, nsteps, stop_time=stop_time)
    return ref, t, dts
