"""Multi-level (AMR) advance on the CUDA path against the reference-header oracle's multi-level driver
(oracle/ref_amr.inc), and its invariants.

Both sides run the same fixed hierarchy (refinement ratio 2, subcycling, flux registers with the
five-equation non-conservative alpha1 source or the six-equation phase-energy and alpha1 terms and the
relaxation of the refluxed cells, average-down), the same coarse-fine interpolation and
the reference's own face arithmetic, so the plain FP64 form is compared to the bit (the asserted bound
is the north star's 1e-11 relative L-infinity per field and box). The coarse-fine operations follow
AMReX's documented semantics on both sides; AMReX itself is not in the image, so they are not pinned
by the reference. Also: one level of several boxes equals the single-box level; the composite-grid
totals of mass, momentum and energy are conserved to round-off on a periodic domain; every level's
boxes go through one box-list launch per RK stage; the mixed form's error.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import amr, cases
from helpers import rel_linf
from oracle.oracle import Oracle, have_ref

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _valid(U, lo, hi, dim, ng=3):
    if dim == 2:
        return U[:, 0, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1]
    return U[:, ng:ng + hi[2] - lo[2] + 1, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1]


def _run(case_fn, kw, domain, regions, mgs, steps, extra=None, precision="fp64"):
    phys, dim, inputs, geom, _ = case_fn(**kw)
    inputs = dict(inputs, **{"compas_b200.precision": precision}, **(extra or {}))
    p, g = cb.make_parm(phys, dim, inputs), cb.make_geom(**geom)
    boxes = amr.hierarchy(domain, dim, regions, mgs)
    states = amr.box_states(case_fn, kw, domain, dim, boxes)
    A = cb.Amr(p, g, boxes)
    for b, U in enumerate(states):
        A.upload(b, U)
    A.advance(steps)
    info = A.sync()
    got = [A.download(b) for b in range(len(boxes))]
    dts = A.dts(info.steps)
    launches = A.launches()
    A.close()
    return p, g, dim, boxes, states, got, dts, info, launches


def _compare(p, g, dim, boxes, states, got, dts, steps):
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    ref = [U.copy() for U in states]
    _, dts_ref = Oracle("reference", p, g).amr_advance(boxes, ref, steps)
    np.testing.assert_array_equal(dts, dts_ref)
    worst = np.zeros(ref[0].shape[0])
    for (lev, lo, hi), a, r in zip(boxes, got, ref):
        worst = np.maximum(worst, rel_linf(_valid(a, lo, hi, dim), _valid(r, lo, hi, dim)))
    print(f"{len(boxes)} boxes, {1 + max(b[0] for b in boxes)} levels, {steps} steps: rel Linf per field "
          f"{np.array2string(worst, precision=2)}; bitwise equal: {all(np.array_equal(_valid(a, *b[1:], dim), _valid(r, *b[1:], dim)) for b, a, r in zip(boxes, got, ref))}")
    assert np.all(worst <= TOL), worst


def test_one_level_of_boxes_equals_single_box_level():
    kw = dict(nx=64, ny=32, scheme="WENO5B")
    p, g, dim, boxes, states, got, dts, info, _ = _run(cases.shock_bubble, kw, (64, 32), [], 16, 5)
    phys, _, inputs, geom, U = cases.shock_bubble(**kw)
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(5)
    ref = lv.download()
    lv.close()
    V = cb.valid_view(ref, p, g)
    for (lev, lo, hi), a in zip(boxes, got):
        np.testing.assert_array_equal(_valid(a, lo, hi, dim), V[:, 0, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1])


@pytest.mark.parametrize("case_fn,kw,domain,regions,mgs,steps", [
    (cases.shock_bubble, dict(nx=64, ny=32, scheme="WENO5B"), (64, 32),
     [((40, 16, 0), (95, 47, 0)), ((96, 48, 0), (175, 79, 0))], 32, 4),
    (cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5"), (48, 24), [((24, 8, 0), (71, 39, 0))], 16, 4),
    (cases.advected_disc, dict(n=32), (32, 32), [((16, 16, 0), (47, 47, 0)), ((40, 40, 0), (87, 87, 0))], 16, 5),
    (cases.advected_interface, dict(n=16, dim=3, physics=cb.FIVEEQS), (16, 16, 16),
     [((8, 8, 8), (23, 23, 23))], 8, 3),
    (cases.advected_interface, dict(n=16, dim=2, physics=cb.SIXEQS), (16, 16),
     [((8, 8, 0), (23, 23, 0)), ((24, 24, 0), (39, 39, 0))], 8, 4),
    (cases.advected_interface, dict(n=16, dim=3, physics=cb.SIXEQS), (16, 16, 16),
     [((8, 8, 8), (23, 23, 23))], 8, 3),
    (cases.shock_droplet, dict(n=16), (16, 16, 16), [((8, 8, 8), (23, 23, 23))], 8, 3),
], ids=["bubble3lev_weno5b", "bubble2lev_weno5", "disc3lev_periodic", "sphere2lev_3d", "sixeq_disc3lev_periodic",
        "sixeq_sphere2lev_3d", "sixeq_droplet2lev_3d"])
def test_amr_matches_oracle(case_fn, kw, domain, regions, mgs, steps):
    p, g, dim, boxes, states, got, dts, info, launches = _run(case_fn, kw, domain, regions, mgs, steps)
    assert info.status == 0 and info.steps == steps
    _compare(p, g, dim, boxes, states, got, dts, steps)


def test_amr_composite_conservation_periodic():
    kw = dict(n=32)
    p, g, dim, boxes, states, got, dts, info, _ = _run(
        cases.advected_disc, kw, (32, 32), [((16, 16, 0), (47, 47, 0)), ((40, 40, 0), (87, 87, 0))], 16, 6)
    cov = amr.covered_mask_fn(boxes, 2)
    for c in range(5):  # masses, momenta, total energy
        s0 = amr.composite_sum(states, boxes, 2, 3, c, cov)
        s1 = amr.composite_sum(got, boxes, 2, 3, c, cov)
        print(f"component {c}: composite total relative change {abs(s1 - s0) / abs(s0):.1e}")
        assert abs(s1 - s0) <= 1e-13 * abs(s0)


def test_sixeq_amr_composite_conservation_periodic():
    kw = dict(n=16, dim=2, physics=cb.SIXEQS)
    p, g, dim, boxes, states, got, dts, info, _ = _run(
        cases.advected_interface, kw, (16, 16), [((8, 8, 0), (23, 23, 0)), ((24, 24, 0), (39, 39, 0))], 8, 6)
    assert info.status == 0
    cov = amr.covered_mask_fn(boxes, 2)

    def totals(st):
        s = [amr.composite_sum(st, boxes, 2, 3, c, cov) for c in range(6)]
        return s[:4] + [s[4] + s[5]]  # masses, momenta, total energy

    for c, (s0, s1) in enumerate(zip(totals(states), totals(got))):
        print(f"quantity {c}: composite total relative change {abs(s1 - s0) / abs(s0):.1e}")
        assert abs(s1 - s0) <= 1e-13 * abs(s0)


def test_amr_levels_use_one_list_launch_per_stage():
    # 3 levels x (1 + 2 + 4 substeps) x 3 stages of list launches plus fills, faces, reflux and average-down
    p, g, dim, boxes, states, got, dts, info, launches = _run(
        cases.shock_bubble, dict(nx=64, ny=32, scheme="WENO5B"), (64, 32),
        [((40, 16, 0), (95, 47, 0)), ((96, 48, 0), (175, 79, 0))], 16, 1)
    nbox = len(boxes)
    assert nbox > 10
    stage_launches = 3 * (1 + 2 + 4)
    print(f"{nbox} boxes, {launches} launches in one coarse step ({stage_launches} box-list stage launches)")
    assert launches < 10 * stage_launches + 20


@pytest.mark.parametrize("args", [
    (cases.shock_bubble, dict(nx=64, ny=32, scheme="WENO5B"), (64, 32),
     [((40, 16, 0), (95, 47, 0)), ((96, 48, 0), (175, 79, 0))], 32, 6),
    (cases.shock_droplet, dict(n=16), (16, 16, 16), [((8, 8, 8), (23, 23, 23))], 8, 6),
], ids=["fiveeq_bubble", "sixeq_droplet"])
def test_amr_mixed_error_vs_fp64(args):
    _, _, dim, boxes, _, a, _, ia, _ = _run(*args, precision="mixed")
    _, _, _, _, _, b, _, ib, _ = _run(*args, precision="fp64")
    assert ia.status == 0 and ib.status == 0
    num = np.zeros(a[0].shape[0])
    den = np.zeros(a[0].shape[0])
    for (lev, lo, hi), x, y in zip(boxes, a, b):
        X, Y = _valid(x, lo, hi, dim), _valid(y, lo, hi, dim)
        num += np.abs(X - Y).reshape(X.shape[0], -1).sum(axis=1)
        den += np.abs(Y).reshape(Y.shape[0], -1).sum(axis=1)
    e = num / den
    print("AMR mixed vs FP64 rel L1 per field:", np.array2string(e, precision=2))
    for c in (0, 1, a[0].shape[0] - 1):  # masses and volume fraction
        assert e[c] <= 1e-5, e


@pytest.mark.parametrize("case_fn,kw,domain,regions,mgs,steps,extra", [
    (cases.triple_point, dict(m=8), (56, 24), [((8, 8, 0), (47, 39, 0)), ((24, 24, 0), (71, 55, 0))], 16, 4,
     {"FiniteVolume.Scheme": "MUSCL-MC"}),
    (cases.triple_point, dict(m=8), (56, 24), [((16, 12, 0), (47, 35, 0))], 16, 4, {}),
    (cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5"), (48, 24), [((24, 8, 0), (71, 39, 0))], 16, 4,
     {"FiniteVolume.Scheme": "MUSCL-MC"}),
    (cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5B"), (48, 24), [((24, 8, 0), (71, 39, 0))], 16, 4,
     {"Physics.RiemannSolver": "HLL"}),
    (cases.shock_droplet, dict(n=16), (16, 16, 16), [((8, 8, 8), (23, 23, 23))], 8, 3,
     {"FiniteVolume.Scheme": "WENO3", "Physics.RiemannSolver": "LLF"}),
    (cases.shock_bubble, dict(nx=48, ny=24, scheme="WENO5"), (48, 24), [((24, 8, 0), (71, 39, 0))], 16, 4,
     {"FiniteVolume.Scheme": "WENO3B"}),
    (cases.triple_point, dict(m=8), (56, 24), [((16, 12, 0), (47, 35, 0))], 16, 4,
     {"FiniteVolume.Scheme": "WENO3B"}),
    (cases.shock_bubble, dict(nx=64, ny=32, scheme="WENO5B"), (64, 32),
     [((40, 16, 0), (95, 47, 0)), ((96, 48, 0), (175, 79, 0))], 32, 4, {"amr.Interpolater": "pc_interp"}),
    (cases.shock_droplet, dict(n=16), (16, 16, 16), [((8, 8, 8), (23, 23, 23))], 8, 3,
     {"amr.Interpolater": "pc_interp"}),
], ids=["triple_muscl_mc_3lev", "triple_weno5_2lev", "bubble_muscl_mc", "bubble_hll", "droplet_weno3_llf",
        "bubble_weno3b", "triple_weno3b", "bubble3lev_pc_interp", "droplet2lev_pc_interp"])
def test_amr_schemes_and_nphase_match_oracle(case_fn, kw, domain, regions, mgs, steps, extra):
    """The multi-level advance with the N-phase model (the triple point, as the reference's example runs
    it: MUSCL-MC on a hierarchy), the three-cell schemes, the LLF / HLL Riemann solvers and the
    piecewise-constant coarse-fine interpolation (amr.Interpolater = pc_interp), to the bit."""
    p, g, dim, boxes, states, got, dts, info, launches = _run(case_fn, kw, domain, regions, mgs, steps, extra)
    assert info.status == 0 and info.steps == steps
    _compare(p, g, dim, boxes, states, got, dts, steps)
