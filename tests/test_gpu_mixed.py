"""The mixed-precision form (FP32 reconstruction; FP64 pressure recovery, Riemann solver, stage
accumulation and relaxation) against the FP64 path, which is the reference's arithmetic to the bit.

The bound is the north star's: relative L1 error (sum |a - b| / sum |b|) in the densities and the
volume fraction <= 1e-5 against the FP64 result after the stated steps; every field's error is
printed. Mass, momentum and energy stay conserved to round-off because each face flux is computed
once and used by both neighbouring cells, whatever its precision."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import run_gpu, run_oracle

pytestmark = pytest.mark.gpu

L1_TOL = 1e-5


def rel_l1(a, b):
    return np.array([float(np.abs(a[c] - b[c]).sum() / max(np.abs(b[c]).sum(), 1e-300)) for c in range(a.shape[0])])


def _pair(case_fn, steps, **kw):
    phys, dim, inputs, geom, U = case_fn(**kw)
    g = cb.make_geom(**geom)
    p64 = cb.make_parm(phys, dim, inputs)
    pmx = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    a, ia, _ = run_gpu(pmx, g, U, steps)
    b, ib, _ = run_gpu(p64, g, U, steps)
    assert ia.status == 0 and ib.status == 0
    return p64, g, U, cb.valid_view(a, p64, g), cb.valid_view(b, p64, g)


def _check(p, name, e, idx):
    print(f"{name}: rel L1 per field vs FP64 {np.array2string(e, precision=2)}")
    for c in idx:
        assert e[c] <= L1_TOL, (c, e)


def test_mixed_shock_droplet_3d():
    p, g, U, a, b = _pair(cases.shock_droplet, 20, n=48)
    e = rel_l1(a, b)
    # densities (alpha_k rho_k, k = 1, 2) and the volume fraction
    _check(p, "shock-droplet 48^3 x 20 steps", e, (0, 1, 7))


def test_mixed_advected_disc_config_against_reference():
    """The CPU-runnable configuration (128^2, 200 steps) in mixed precision against the reference's
    own arithmetic (oracle): the equilibrium of uniform p and u must survive the FP32 reconstruction."""
    phys, dim, inputs, geom, U = cases.advected_disc(n=128)
    g = cb.make_geom(**geom)
    pmx = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    p64 = cb.make_parm(phys, dim, inputs)
    got, info, _ = run_gpu(pmx, g, U, 200)
    ref, t, _ = run_oracle(p64, g, U, 200)
    a, r = cb.valid_view(got, p64, g), cb.valid_view(ref, p64, g)
    e = rel_l1(a, r)
    _check(p64, "advected disc 128^2 x 200 steps", e, (0, 1, 5))
    rho = a[0] + a[1]
    u = a[2] / rho
    assert np.max(np.abs(u - 1.0)) < 1e-6


def test_mixed_weno5b_bubble():
    p, g, U, a, b = _pair(cases.shock_bubble, 30, nx=128, ny=64, scheme="WENO5B")
    e = rel_l1(a, b)
    _check(p, "shock-bubble WENO5B 128x64 x 30 steps", e, (0, 1, 5))
    assert a[5].min() >= -1e-12 and a[5].max() <= 1 + 1e-12


def test_mixed_conserves_to_round_off():
    phys, dim, inputs, geom, U = cases.advected_disc(n=64)
    g = cb.make_geom(**geom)
    pmx = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    got, info, _ = run_gpu(pmx, g, U, 50)
    V0, V = cb.valid_view(U, pmx, g), cb.valid_view(got, pmx, g)
    for c in range(5):
        s0 = float(V0[c].sum())
        assert abs(float(V[c].sum()) - s0) <= 1e-12 * float(np.abs(V0[c]).sum()), c
