"""GODUNOV, the MUSCL family and WENO3 (FiniteVolume.Scheme = GODUNOV, MUSCL, MUSCL-Minmod, MUSCL-vanLeer,
MUSCL-Superbee, MUSCL-MC, WENO3, WENO3B) on the CUDA path against the reference-header oracle: the plain FP64 form
is compared to the bit over several steps for every limiter (five-equation 2D), the six-equation 3D
droplet with relaxation, and the N-phase triple point with the scheme of the reference's own example
(exec/TriplePoint-5Eq-N/prob/inputs: MUSCL-MC, followed by the consistent limiter); the LLF and HLL
Riemann solvers (Physics.RiemannSolver) likewise; and the mixed form's error against the FP64 form."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import rel_linf, run_gpu, run_oracle
from oracle.oracle import have_ref

pytestmark = pytest.mark.gpu

SCHEMES = ["GODUNOV", "MUSCL", "MUSCL-vanLeer", "MUSCL-Superbee", "MUSCL-MC", "WENO3", "WENO3B"]


def _run(fn, kw, scheme, nsteps, prec="fp64"):
    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": scheme, "compas_b200.precision": prec}))
    g = cb.make_geom(**geom)
    return p, g, U


def _bitwise(p, g, U, nsteps):
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    got, info, dts = run_gpu(p, g, U, nsteps)
    ref, _, dts_ref = run_oracle(p, g, U, nsteps, kind="reference")
    assert info.status == 0 and info.steps == nsteps
    np.testing.assert_array_equal(dts, dts_ref)
    e = rel_linf(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    print(f"{nsteps} steps, rel Linf per field {np.array2string(e, precision=2)}")
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))


@pytest.mark.parametrize("scheme", SCHEMES)
def test_fiveeq_2d_bitwise(scheme):
    p, g, U = _run(cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5"), scheme, 6)
    _bitwise(p, g, U, 6)


@pytest.mark.parametrize("scheme", ["MUSCL-MC", "MUSCL-Superbee", "WENO3", "WENO3B"])
def test_sixeq_3d_droplet_bitwise(scheme):
    p, g, U = _run(cases.shock_droplet, dict(n=16), scheme, 4)
    _bitwise(p, g, U, 4)


@pytest.mark.parametrize("scheme", ["MUSCL-MC", "GODUNOV", "WENO3", "WENO3B"])
def test_triple_point_bitwise(scheme):
    p, g, U = _run(cases.triple_point, dict(m=12), scheme, 6)
    _bitwise(p, g, U, 6)


@pytest.mark.parametrize("scheme", ["MUSCL-MC", "WENO3", "WENO3B"])
@pytest.mark.parametrize("fn,kw", [(cases.shock_bubble, dict(nx=64, ny=32, scheme="WENO5")),
                                   (cases.shock_droplet, dict(n=24))], ids=["bubble", "droplet"])
def test_mixed_error_vs_fp64(fn, kw, scheme):
    out = {}
    for prec in ("fp64", "mixed"):
        p, g, U = _run(fn, kw, scheme, 10, prec)
        got, info, _ = run_gpu(p, g, U, 10)
        assert info.status == 0
        out[prec] = cb.valid_view(got, p, g)
    A, B = out["mixed"], out["fp64"]
    e = np.array([float(np.abs(A[c] - B[c]).sum() / np.abs(B[c]).sum()) for c in range(A.shape[0])])
    print(f"{scheme} mixed vs FP64 rel L1 per field:", np.array2string(e, precision=2))
    np_ = p.nphase if p.physics == cb.FIVEEQS_NPHASE else 2
    masses = list(range(np_))
    alphas = list(range(A.shape[0] - (np_ if p.physics == cb.FIVEEQS_NPHASE else 1), A.shape[0]))
    for c in masses + alphas:
        assert e[c] <= 1e-5, e


def test_triple_point_mixed_error_within_fp64_sensitivity():
    """The triple point starts from sharp interfaces, where the MC limiter switches branch on a
    rounding-level change of its slopes, so the mixed form is held to 10x the FP64 form's own change
    under a relative 2^-24 perturbation (random sign per value) of the initial state, over 10 steps."""
    p64, g, U = _run(cases.triple_point, dict(m=16), "MUSCL-MC", 10)
    pmx, _, _ = _run(cases.triple_point, dict(m=16), "MUSCL-MC", 10, "mixed")
    a, ia, _ = run_gpu(pmx, g, U.copy(), 10)
    b, ib, _ = run_gpu(p64, g, U.copy(), 10)
    rng = np.random.default_rng(0)
    Up = U * (1.0 + 2.0 ** -24 * rng.choice([-1.0, 1.0], size=U.shape))
    c, ic, _ = run_gpu(p64, g, Up, 10)
    assert ia.status == 0 and ib.status == 0 and ic.status == 0
    X, Y, Z = (cb.valid_view(v, p64, g) for v in (a, b, c))

    def rel_l1(P, Q):
        return np.array([float(np.abs(P[k] - Q[k]).sum() / np.abs(Q[k]).sum()) for k in range(P.shape[0])])

    e, sens = rel_l1(X, Y), rel_l1(Z, Y)
    print("triple point MUSCL-MC mixed vs FP64 rel L1:", np.array2string(e, precision=2),
          "FP64 sensitivity:", np.array2string(sens, precision=2))
    for k in (0, 1, 2, 6, 7, 8):  # partial densities and volume fractions
        assert e[k] <= 10.0 * sens[k], (e, sens)


@pytest.mark.parametrize("solver", ["LLF", "HLL"])
@pytest.mark.parametrize("fn,kw,scheme,nsteps", [
    (cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5B"), "WENO5B", 5),
    (cases.shock_droplet, dict(n=16), "WENO5", 3),
    (cases.triple_point, dict(m=12), "MUSCL-MC", 5),
], ids=["bubble_weno5b", "droplet_weno5", "triple_muscl_mc"])
def test_llf_hll_bitwise(solver, fn, kw, scheme, nsteps):
    """Physics.RiemannSolver = LLF and HLL (the five-equation, six-equation and N-phase forms with their
    face velocities and, for the six-equation model, the face values of u alpha_k p_k), FP64 against the
    reference headers to the bit."""
    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": scheme, "Physics.RiemannSolver": solver}))
    g = cb.make_geom(**geom)
    _bitwise(p, g, U, nsteps)


@pytest.mark.parametrize("solver", ["LLF", "HLL"])
def test_llf_hll_mixed_error_vs_fp64(solver):
    out = {}
    for prec in ("fp64", "mixed"):
        phys, dim, inputs, geom, U = cases.shock_droplet(n=24)
        p = cb.make_parm(phys, dim, dict(inputs, **{"Physics.RiemannSolver": solver, "compas_b200.precision": prec}))
        g = cb.make_geom(**geom)
        got, info, _ = run_gpu(p, g, U, 10)
        assert info.status == 0
        out[prec] = cb.valid_view(got, p, g)
    A, B = out["mixed"], out["fp64"]
    e = np.array([float(np.abs(A[c] - B[c]).sum() / np.abs(B[c]).sum()) for c in range(A.shape[0])])
    print(f"{solver} mixed vs FP64 rel L1 per field:", np.array2string(e, precision=2))
    for c in (0, 1, A.shape[0] - 1):
        assert e[c] <= 1e-5, e


@pytest.mark.parametrize("fn,kw,nsteps", [
    (cases.triple_point, dict(m=12), 6),
    (cases.nphase_bubbles, dict(n=24, nphase=4), 4),
    (cases.nphase_bubbles, dict(n=10, nphase=3, dim=3), 3),
], ids=["triple", "bubbles_np4", "bubbles3d_np3"])
def test_nphase_weno5b_bitwise(fn, kw, nsteps):
    """FiniteVolume.Scheme = WENO5B for the N-phase model: per-phase bounded reconstruction of alpha_k
    rho_k and alpha_k with the partial densities' weights, renormalisation, the second limiting pass
    (FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq_NPhase.H), to the bit."""
    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": "WENO5B"}))
    g = cb.make_geom(**geom)
    _bitwise(p, g, U, nsteps)


def test_nphase_weno5b_mixed_error_vs_fp64():
    out = {}
    for prec in ("fp64", "mixed"):
        phys, dim, inputs, geom, U = cases.nphase_bubbles(n=32, nphase=3)
        p = cb.make_parm(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": "WENO5B", "compas_b200.precision": prec}))
        g = cb.make_geom(**geom)
        got, info, _ = run_gpu(p, g, U, 10)
        assert info.status == 0
        out[prec] = cb.valid_view(got, p, g)
    A, B = out["mixed"], out["fp64"]
    e = np.array([float(np.abs(A[c] - B[c]).sum() / np.abs(B[c]).sum()) for c in range(A.shape[0])])
    print("N-phase WENO5B mixed vs FP64 rel L1 per field:", np.array2string(e, precision=2))
    for c in (0, 1, 2, A.shape[0] - 3, A.shape[0] - 2, A.shape[0] - 1):
        assert e[c] <= 1e-5, e
