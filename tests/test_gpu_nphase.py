"""The N-phase five-equation model (FIVEEQS_NPHASE) on the CUDA path against the CPU oracles.

The plain FP64 form reproduces the reference's arithmetic - WENO5 in primitive variables, the
consistent limiter of the partial densities and volume fractions, HLLC, the Kapila terms of every
volume fraction - so the right-hand side, the face wave speed and whole level advances are compared
to the bit against the reference-header oracle (the asserted bound is the north star's 1e-11
relative L-infinity per field). Cases: the triple point of the serving workload (NPHASE = 3, sharp
interfaces, reflecting walls), advected bubbles with 2, 3 and 4 phases, the Kapila K term and the
NASG covolume, a 3D case; the box-list (batched) form against the single-box form; and the mixed
form's error against FP64.
"""
import ast
import glob
import os

import numpy as np
import pytest
import torch

import compas_b200 as cb
from compas_b200 import cases
from helpers import oracle_kind, rel_linf, run_gpu, run_oracle
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _case(fn, **kw):
    phys, dim, inputs, geom, U = fn(**kw)
    return cb.make_parm(phys, dim, inputs), cb.make_geom(**geom), U


CASES = [
    (cases.triple_point, dict(m=8)),
    (cases.triple_point, dict(m=16, gammas=cases.TRIPLE_POINT_REFERENCE_GAMMAS)),
    (cases.nphase_bubbles, dict(n=40, nphase=2)),
    (cases.nphase_bubbles, dict(n=40, nphase=3, source_term=1)),
    (cases.nphase_bubbles, dict(n=32, nphase=4, eos=3, source_term=1)),
    (cases.nphase_bubbles, dict(n=16, nphase=3, dim=3)),
]
IDS = ["triple8", "triple16_refgamma", "bubbles2", "bubbles3_K", "bubbles4_nasg_K", "bubbles3_3d"]
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*5eqn*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_nphase_matches_reference_golden(path):
    """Fixtures made by the reference's own N-phase headers (tests/golden/make_golden.py)."""
    z = np.load(path)
    phys, dim, steps = (int(x) for x in z["physics"])
    p = cb.make_parm(phys, dim, ast.literal_eval(str(z["inputs"])))
    g = cb.make_geom(**ast.literal_eval(str(z["geom"])))
    got, info, dts = run_gpu(p, g, z["U0"].copy(), steps)
    assert info.status == 0 and info.steps == steps
    e = rel_linf(cb.valid_view(got, p, g), z["valid"])
    print(f"{os.path.basename(path)}: rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(cb.valid_view(got, p, g), z['valid'])}")
    np.testing.assert_array_equal(dts, z["dts"])
    assert np.all(e <= TOL), e



@pytest.mark.parametrize("fn,kw", CASES, ids=IDS)
def test_nphase_dudt_matches_oracle(fn, kw):
    p, g, U = _case(fn, **kw)
    o = Oracle(oracle_kind(p.physics, p.dim, p.nphase), p, g)
    ref = U.copy()
    o.fill_ghosts(ref)
    dref, cref = o.compute_dudt(ref)
    dev = torch.device("cuda")
    Ud = torch.from_numpy(ref).to(dev)
    dU = torch.zeros_like(Ud)
    cm = torch.zeros(1, dtype=torch.float64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    cb.compute_dUdt_FV(p, g, Ud, dU, cm, err)
    torch.cuda.synchronize()
    got = dU.cpu().numpy()
    e = rel_linf(cb.valid_view(got, p, g), cb.valid_view(dref, p, g))
    print(f"{o.kind} oracle: dUdt rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(cb.valid_view(got, p, g), cb.valid_view(dref, p, g))}; "
          f"cmax {float(cm.item())!r} vs {cref!r}")
    assert int(err.item()) == 0
    assert np.all(e <= TOL), e
    assert float(cm.item()) == cref


@pytest.mark.parametrize("fn,kw,steps", [(f, k, s) for (f, k), s in zip(CASES, [40, 20, 30, 30, 20, 6])], ids=IDS)
def test_nphase_advance_matches_oracle(fn, kw, steps):
    p, g, U = _case(fn, **kw)
    got, info, dts = run_gpu(p, g, U.copy(), steps)
    assert info.status == 0 and info.steps == steps
    ref, t, dts_ref = run_oracle(p, g, U, steps)
    e = rel_linf(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    print(f"{steps} steps: rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))}")
    np.testing.assert_array_equal(dts, dts_ref)
    assert np.all(e <= TOL), e


def test_nphase_volume_fractions_sum_and_walls():
    """Triple point: the volume fractions keep summing to 1 to round-off, the walls keep the total
    mass of every material, and nothing crosses the reflecting walls."""
    p, g, U = _case(cases.triple_point, m=16)
    got, info, _ = run_gpu(p, g, U.copy(), 60)
    assert info.status == 0
    V0, V1 = cb.valid_view(U, p, g), cb.valid_view(got, p, g)
    s = V1[6] + V1[7] + V1[8]
    print(f"sum of volume fractions in [{s.min()!r}, {s.max()!r}]")
    assert np.all(np.abs(s - 1.0) < 1e-11)
    for k in range(3):
        m0, m1 = V0[k].sum(), V1[k].sum()
        print(f"material {k + 1}: relative mass change {abs(m1 - m0) / m0:.1e}")
        assert abs(m1 - m0) <= 1e-12 * m0


def test_nphase_batch_equals_level():
    """Cases of different sizes in one box-list batch give the single-box level's bits."""
    reqs = [dict(m=8), dict(m=12), dict(m=16, gammas=cases.TRIPLE_POINT_REFERENCE_GAMMAS)]
    b = cb.Batch(cb.FIVEEQS_NPHASE, 2, id_limiter=5, precision=0, capacity=8, nphase=3)
    ids, ins = [], []
    for kw in reqs:
        p, g, U = _case(cases.triple_point, **kw)
        ids.append(b.add(p, g, U, max_steps=25))
        ins.append((p, g, U))
    b.advance(25)
    for cid, (p, g, U) in zip(ids, ins):
        got = b.download(cid)
        ref, info, _ = run_gpu(p, g, U.copy(), 25)
        assert np.array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    b.close()


def _rel_l1(X, Y):
    return np.abs(X - Y).reshape(X.shape[0], -1).sum(axis=1) / np.abs(Y).reshape(Y.shape[0], -1).sum(axis=1)


def test_nphase_mixed_error_vs_fp64():
    """Mixed form against FP64 on the triple point. Over 10 steps the relative L1 error of the partial
    densities and volume fractions is held to 1e-5. Over 100 steps the shear layer at the triple point
    amplifies any rounding difference, so the bound there is 10x the FP64 form's own change when its
    initial state is perturbed at FP32 rounding level (a relative 2^-24 of random sign per value)."""
    phys, dim, inputs, geom, U = cases.triple_point(m=32)
    g = cb.make_geom(**geom)
    pm = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    pf = cb.make_parm(phys, dim, inputs)
    for steps in (10, 100):
        a, ia, _ = run_gpu(pm, g, U.copy(), steps)
        b, ib, _ = run_gpu(pf, g, U.copy(), steps)
        assert ia.status == 0 and ib.status == 0
        X, Y = cb.valid_view(a, pf, g), cb.valid_view(b, pf, g)
        e = _rel_l1(X, Y)
        print(f"triple point, {steps} steps: mixed vs FP64 rel L1 per field {np.array2string(e, precision=2)}")
        comps = (0, 1, 2, 6, 7, 8)
        if steps == 10:
            for c in comps:
                assert e[c] <= 1e-5, e
        else:
            rng = np.random.Generator(np.random.PCG64(7))
            Up = U * (1.0 + 2.0 ** -24 * rng.choice([-1.0, 1.0], size=U.shape))
            c_, ic, _ = run_gpu(pf, g, Up, steps)
            assert ic.status == 0
            sens = _rel_l1(cb.valid_view(c_, pf, g), Y)
            print(f"FP64 change under an FP32-level perturbation of the initial state: "
                  f"{np.array2string(sens, precision=2)}")
            for c in comps:
                assert e[c] <= 10.0 * sens[c], (e, sens)
