"""The N-phase six-equation model in its internal-energy form (SIXEQS_IE_NPHASE) on the CUDA path
against the reference's own headers.

The model's plain FP64 form reproduces the reference's arithmetic: the phase pressures from the
phase internal energies, reconstruction in primitive variables (GODUNOV, MUSCL with the consistent
limiter of volume fractions, partial densities and phase pressures, WENO3, WENO3B, WENO5, WENO5B with
bounded partial densities and volume fractions), the model's HLLC / HLL / LLF fluxes, the
non-conservative terms alpha_k div u and alpha_k p_k div u, and the Newton pressure relaxation with its
safeguarded fallback after every stage. The right-hand side, the face wave speed and whole level
advances are compared to the bit against the reference-header oracle (oracle/_ref/libref_6eqn*); the
asserted bound is the north star's 1e-11 relative L-infinity per field. Cases: a Mach 1.1 water shock
on an air bubble (and a helium bubble with three phases), after the reference's
ShockBubble-WaterAir-6Eq-Nphase example, in pressure equilibrium and out of it, with the NASG
covolume, with a trace threshold that sends phases through the safeguarded relaxation, and in 3D.
The mixed form (FP32 reconstruction) is held to 1e-5 relative L1 against the FP64 form in the volume
fractions and phase masses with the WENO schemes (1e-3 with MUSCL, whose discontinuous limiter turns
rounding into branch flips), and its box-list batch to the bits of its single-box level.
"""
import ast
import glob
import os

import numpy as np
import pytest
import torch

import compas_b200 as cb
from compas_b200 import cases
from helpers import rel_linf, run_gpu
from oracle.oracle import Oracle, have_ref

pytestmark = pytest.mark.gpu

TOL = 1e-11

SCHEMES = ["GODUNOV", "MUSCL", "MUSCL-vanLeer", "MUSCL-MC", "WENO3", "WENO3B", "WENO5", "WENO5B"]
RIEMANN = ["HLLC", "HLL", "LLF"]

CASES = {
    "np2": dict(n=16, nphase=2),
    "np3_dp": dict(n=16, nphase=3, dp=0.05),
    "np2_nasg_dp": dict(n=16, nphase=2, eos=3, dp=0.05),
    "np3_trace": dict(n=16, nphase=3, dp=0.05, trace=1e-3),
    "np3_3d": dict(n=8, nphase=3, dim=3, dp=0.05),
}


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*_6eqn*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_sixn_matches_reference_golden(path):
    """Fixtures made by the reference's own SIXEQS_IE_NPHASE headers (tests/golden/make_golden.py)."""
    z = np.load(path)
    phys, dim, steps = (int(x) for x in z["physics"])
    p = cb.make_parm(phys, dim, ast.literal_eval(str(z["inputs"])))
    g = cb.make_geom(**ast.literal_eval(str(z["geom"])))
    got, info, dts = run_gpu(p, g, z["U0"].copy(), steps)
    assert info.status == 0 and info.steps == steps
    a = cb.valid_view(got, p, g)
    e = rel_linf(a, z["valid"])
    print(f"{os.path.basename(path)}: rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(a, z['valid'])}")
    np.testing.assert_array_equal(dts, z["dts"])
    assert np.all(e <= TOL), e


def _case(**kw):
    phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(**kw)
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("the SIXEQS_IE_NPHASE oracle is the reference build (oracle/_ref/libref_6eqn*)")
    return p, g, U


def _dudt_pair(p, g, U):
    o = Oracle("reference", p, g)
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
    return dU.cpu().numpy(), float(cm.item()), int(err.item()), dref, cref


@pytest.mark.parametrize("riemann", RIEMANN)
@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("name", ["np2", "np3_dp", "np3_3d"])
def test_sixn_dudt_matches_reference(name, scheme, riemann):
    p, g, U = _case(**CASES[name], scheme=scheme, riemann=riemann)
    got, cm, err, dref, cref = _dudt_pair(p, g, U)
    a, b = cb.valid_view(got, p, g), cb.valid_view(dref, p, g)
    e = rel_linf(a, b)
    print(f"{name} {scheme} {riemann}: dUdt rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(a, b)}; cmax {cm!r} vs {cref!r}")
    assert err == 0
    assert np.all(e <= TOL), e
    assert cm == cref


@pytest.mark.parametrize("scheme", ["MUSCL", "WENO5", "WENO5B"])
def test_sixn_dudt_nasg(scheme):
    p, g, U = _case(**CASES["np2_nasg_dp"], scheme=scheme)
    got, cm, err, dref, cref = _dudt_pair(p, g, U)
    e = rel_linf(cb.valid_view(got, p, g), cb.valid_view(dref, p, g))
    print(f"NASG {scheme}: rel Linf per field {np.array2string(e, precision=2)}")
    assert err == 0
    assert np.all(e <= TOL), e
    assert cm == cref


ADVANCES = [
    ("np2", "MUSCL", "HLLC", 30),
    ("np3_dp", "MUSCL", "HLLC", 25),
    ("np3_dp", "WENO5B", "HLLC", 20),
    ("np3_dp", "WENO5", "LLF", 20),
    ("np2_nasg_dp", "MUSCL-MC", "HLL", 20),
    ("np3_trace", "WENO3B", "HLLC", 20),
    ("np3_3d", "MUSCL", "HLLC", 6),
]


@pytest.mark.parametrize("name,scheme,riemann,steps", ADVANCES,
                         ids=[f"{a}-{b}-{c}" for a, b, c, _ in ADVANCES])
def test_sixn_advance_matches_reference(name, scheme, riemann, steps):
    """TVD-RK3 steps with the pressure relaxation after every stage and the CFL time step."""
    p, g, U = _case(**CASES[name], scheme=scheme, riemann=riemann)
    got, info, dts = run_gpu(p, g, U.copy(), steps)
    assert info.status == 0 and info.steps == steps
    ref = U.copy()
    t, dts_ref = Oracle("reference", p, g).advance(ref, steps)
    a, b = cb.valid_view(got, p, g), cb.valid_view(ref, p, g)
    e = rel_linf(a, b)
    print(f"{name} {scheme} {riemann}, {steps} steps: rel Linf per field {np.array2string(e, precision=2)}; "
          f"bitwise equal: {np.array_equal(a, b)}")
    np.testing.assert_array_equal(dts, dts_ref)
    assert np.all(e <= TOL), e


def test_sixn_relaxation_equalises_phase_pressures():
    """After an advance with relaxation every phase with volume fraction above the trace threshold
    carries the mixture pressure: alpha_k p_k / alpha_k agrees across the phases."""
    p, g, U = _case(**CASES["np3_dp"], scheme="MUSCL")
    got, info, _ = run_gpu(p, g, U.copy(), 5)
    assert info.status == 0
    V = cb.valid_view(got, p, g)
    npk = p.nphase
    A = np.array(p.Ak[:npk])
    B = np.array(p.Bk[:npk])
    al = V[0:npk]
    are = V[2 * npk:3 * npk]
    pk = (are - al * B[:, None, None, None]) / (A[:, None, None, None] * al)
    mask = np.all(al > 1e-3, axis=0)
    spread = np.max(np.abs(pk[:, mask] - pk[0:1, mask]) / np.abs(pk[0:1, mask]))
    print(f"largest relative spread of the phase pressures over {int(mask.sum())} mixed cells: {spread:.2e}")
    assert spread < 1e-9
    assert np.allclose(al.sum(axis=0), 1.0, atol=1e-12, rtol=0)


def test_sixn_conservation():
    """Masses, momentum and total energy change only through the boundary fluxes: on a periodic
    box the totals stay to round-off."""
    phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(n=16, nphase=3, dp=0.05)
    geom = dict(geom, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    got, info, _ = run_gpu(p, g, U.copy(), 20)
    assert info.status == 0
    a, b = cb.valid_view(got, p, g), cb.valid_view(U, p, g)
    npk = p.nphase
    cons = list(range(npk, 2 * npk)) + list(range(3 * npk, 3 * npk + dim + 1))
    for c in cons:
        s0, s1 = float(b[c].sum()), float(a[c].sum())
        scale = float(np.abs(b[c]).sum())
        print(f"component {c}: total {s0!r} -> {s1!r}")
        assert abs(s1 - s0) <= 1e-13 * scale


def test_sixn_batch_equals_level():
    """Cases of different sizes in one box-list batch give the single-box level's bits."""
    reqs = [dict(n=8, nphase=2), dict(n=12, nphase=2, dp=0.05), dict(n=16, nphase=2, scheme="WENO5")]
    b = cb.Batch(cb.SIXEQS_IE_NPHASE, 2, id_limiter=5, precision=0, capacity=4, nphase=2)
    ids, ins = [], []
    for kw in reqs:
        kw = dict(kw, scheme="WENO5")
        phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(**kw)
        p, g = cb.make_parm(phys, dim, inputs), cb.make_geom(**geom)
        ids.append(b.add(p, g, U, max_steps=12))
        ins.append((p, g, U))
    b.advance(12)
    for cid, (p, g, U) in zip(ids, ins):
        got = b.download(cid)
        ref, info, _ = run_gpu(p, g, U.copy(), 12)
        assert np.array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    b.close()


@pytest.mark.parametrize("scheme", ["MUSCL", "WENO5B"])
def test_sixn_face_flux_divergence_is_the_fused_right_hand_side(scheme):
    """The area-unscaled face fluxes of compas_b200_face_fluxes difference to the conservative part of
    the fused right-hand side (masses and momenta) bit for bit."""
    phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(n=12, nphase=3, dp=0.05, scheme=scheme)
    p, g = cb.make_parm(phys, dim, inputs), cb.make_geom(**geom)
    Ud = torch.from_numpy(U).cuda()
    cb.FillPatch(p, g, Ud)
    dU = torch.zeros_like(Ud)
    cb.compute_dUdt_FV(p, g, Ud, dU)
    N, NC = cb.parm_nstate(p), cb.nc_terms(p)
    F = [torch.zeros(cb.face_shape(p, g, d, N), dtype=torch.float64, device="cuda") for d in range(dim)]
    Fn = [torch.zeros(cb.face_shape(p, g, d, NC), dtype=torch.float64, device="cuda") for d in range(dim)]
    cb.face_fluxes(p, g, Ud, F, Fn, area_scaled=False)
    torch.cuda.synchronize()
    F = [f.cpu().numpy() for f in F]
    acc = None
    for d in range(dim):
        df = F[d][:, :, :, 1:] - F[d][:, :, :, :-1] if d == 0 else F[d][:, :, 1:, :] - F[d][:, :, :-1, :]
        t = df / g.dx[d]
        acc = t if acc is None else acc + t
    got = cb.valid_view(dU.cpu().numpy(), p, g)
    npk = p.nphase
    for c in list(range(npk, 2 * npk)) + list(range(3 * npk, 3 * npk + dim)):
        np.testing.assert_array_equal(-acc[c], got[c], err_msg=f"component {c}")


def _amr_run(kw, domain, regions, mgs, steps, extra=None):
    from compas_b200 import amr
    phys, dim, inputs, geom, _ = cases.sixn_shock_bubbles(**kw)
    p, g = cb.make_parm(phys, dim, dict(inputs, **(extra or {}))), cb.make_geom(**geom)
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("the SIXEQS_IE_NPHASE oracle is the reference build (oracle/_ref/libref_6eqn*)")
    boxes = amr.hierarchy(domain, dim, regions, mgs)
    states = amr.box_states(cases.sixn_shock_bubbles, kw, domain, dim, boxes)
    A = cb.Amr(p, g, boxes)
    for b, U in enumerate(states):
        A.upload(b, U)
    A.advance(steps)
    info = A.sync()
    got = [A.download(b) for b in range(len(boxes))]
    dts = A.dts(info.steps)
    A.close()
    assert info.status == 0 and info.steps == steps
    ref = [U.copy() for U in states]
    _, dts_ref = Oracle("reference", p, g).amr_advance(boxes, ref, steps)
    np.testing.assert_array_equal(dts, dts_ref)
    ng = geom["ng"]
    worst = np.zeros(ref[0].shape[0])
    equal = True
    for (lev, lo, hi), a, r in zip(boxes, got, ref):
        if dim == 2:
            sl = (slice(None), 0, slice(ng, ng + hi[1] - lo[1] + 1), slice(ng, ng + hi[0] - lo[0] + 1))
        else:
            sl = (slice(None), slice(ng, ng + hi[2] - lo[2] + 1), slice(ng, ng + hi[1] - lo[1] + 1),
                  slice(ng, ng + hi[0] - lo[0] + 1))
        worst = np.maximum(worst, rel_linf(a[sl], r[sl]))
        equal = equal and np.array_equal(a[sl], r[sl])
    print(f"{len(boxes)} boxes, {1 + max(b[0] for b in boxes)} levels, {steps} steps: rel Linf per field "
          f"{np.array2string(worst, precision=2)}; bitwise equal: {equal}")
    assert np.all(worst <= TOL), worst


AMR_CASES = [
    (dict(n=16, nphase=2, dp=0.05), (32, 16), [((8, 4, 0), (47, 27, 0))], 16, 4, {}),
    (dict(n=16, nphase=2, dp=0.05), (32, 16), [((8, 4, 0), (47, 27, 0))], 16, 4, {"amr.Interpolater": "pc_interp"}),
    (dict(n=16, nphase=3, dp=0.05, scheme="WENO5B"), (32, 16),
     [((8, 4, 0), (55, 27, 0)), ((32, 16, 0), (79, 47, 0))], 16, 3, {}),
    (dict(n=8, nphase=3, dim=3, dp=0.05), (16, 8, 8), [((8, 4, 4), (23, 11, 11))], 8, 2, {}),
]


@pytest.mark.parametrize("kw,domain,regions,mgs,steps,extra", AMR_CASES,
                         ids=["np2_muscl_2lev", "np2_muscl_2lev_pc_interp", "np3_weno5b_3lev", "np3_muscl_3d_2lev"])
def test_sixn_amr_matches_reference(kw, domain, regions, mgs, steps, extra):
    """The multi-level advance of the model (the reference's ShockBubble-WaterAir-6Eq-Nphase example runs
    it on a hierarchy): subcycling, flux registers with the alpha_k and alpha_k p_k reflux source terms,
    the relaxation of the refluxed cells, average-down; to the bit against the oracle's hierarchy driver."""
    _amr_run(kw, domain, regions, mgs, steps, extra)


def _rel_l1(a, b):
    return np.array([float(np.abs(a[c] - b[c]).sum()) / max(float(np.abs(b[c]).sum()), 1e-300)
                     for c in range(a.shape[0])])


@pytest.mark.parametrize("kw,steps,bound", [
    (dict(n=64, nphase=2, scheme="WENO5"), 40, 1e-5),
    (dict(n=32, nphase=3, dim=3, scheme="WENO5B"), 20, 1e-5),
    # MUSCL's limiter is discontinuous: FP32 rounding of the slopes flips its branch choices, and the
    # out-of-equilibrium three-phase bubble carries that further (measured 2.3e-4 after 40 steps)
    (dict(n=64, nphase=3, dp=0.05, scheme="MUSCL"), 40, 1e-3),
])
def test_sixn_mixed_error_vs_fp64(kw, steps, bound):
    """The mixed form of SIXEQS_IE_NPHASE (FP32 reconstruction of the primitives; FP64 phase-pressure
    recovery, consistent limiter, Riemann solver, relaxation and stage accumulation): relative L1 error
    per field against the FP64 form after the stated steps (each form with its own step sizes), bounded
    on the volume fractions and the phase masses: 1e-5 with the WENO schemes."""
    phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(**kw)
    g = cb.make_geom(**geom)
    out = {}
    for prec in ("fp64", "mixed"):
        p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec}))
        got, info, _ = run_gpu(p, g, U.copy(), steps)
        assert info.status == 0 and info.steps == steps
        out[prec] = cb.valid_view(got, p, g)
    e = _rel_l1(out["mixed"], out["fp64"])
    nph = kw["nphase"]
    print(f"SIXEQS_IE_NPHASE mixed vs FP64 {kw}, {steps} steps: rel L1 per field {np.array2string(e, precision=2)}")
    assert np.all(e[:2 * nph] <= bound), e  # alpha_k then alpha_k rho_k
    assert np.all(np.isfinite(out["mixed"]))


def test_sixn_mixed_batch_equals_level():
    """In the mixed form too, cases in one box-list batch give the single-box level's bits."""
    reqs = [dict(n=8, nphase=2), dict(n=12, nphase=2, dp=0.05), dict(n=16, nphase=2)]
    b = cb.Batch(cb.SIXEQS_IE_NPHASE, 2, id_limiter=5, precision=1, capacity=4, nphase=2)
    ids, ins = [], []
    for kw in reqs:
        phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(**dict(kw, scheme="WENO5"))
        p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
        g = cb.make_geom(**geom)
        ids.append(b.add(p, g, U, max_steps=10))
        ins.append((p, g, U))
    b.advance(10)
    for cid, (p, g, U) in zip(ids, ins):
        got = b.download(cid)
        ref, info, _ = run_gpu(p, g, U.copy(), 10)
        assert info.status == 0
        assert np.array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    b.close()
