"""Refinement tagging and regrid of the multi-level object on the device (compas_b200_amr_tag,
compas_b200_amr_regrid, with the host clustering compas_b200.amr.regrid_boxes).

  * the tags of a level of several boxes equal those of the same state on one box (the ghost cells of a
    level come from its neighbours exactly as a single box's interior);
  * a regrid keeps level 0 to the bit, copies the fine cells that stay refined to the bit, fills the
    newly refined cells by the cell-conservative interpolation of the coarse level (the mean of the
    children of a coarse cell equals it), and so keeps the composite totals of the conserved
    components; the advance then continues from the new hierarchy;
  * a shock-bubble run that regrids every few steps keeps its fine level on the tagged cells.
The clustering is this engine's own (blocks of the blocking factor, greedy growth); AMReX's
Berger-Rigoutsos clustering is not restated, so box layouts are not compared with the reference's.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import amr, cases

pytestmark = pytest.mark.gpu

NG = 3


def _valid(U, lo, hi, dim):
    if dim == 2:
        return U[:, 0, NG:NG + hi[1] - lo[1] + 1, NG:NG + hi[0] - lo[0] + 1]
    return U[:, NG:NG + hi[2] - lo[2] + 1, NG:NG + hi[1] - lo[1] + 1, NG:NG + hi[0] - lo[0] + 1]


def _bubble_amr(nx=128, ny=64, regions=(((48, 32, 0), (143, 95, 0)),), mgs=32, periodic=False, precision="fp64"):
    kw = dict(nx=nx, ny=ny, scheme="WENO5B")
    phys, dim, inputs, geom, _ = cases.shock_bubble(**kw, quadrature=False)
    if periodic:
        geom = dict(geom, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": precision}))
    g = cb.make_geom(**geom)
    boxes = amr.hierarchy((nx, ny), dim, list(regions), mgs)
    states = amr.box_states(cases.shock_bubble, kw, (nx, ny), dim, boxes)
    A = cb.Amr(p, g, boxes)
    for b, U in enumerate(states):
        A.upload(b, U)
    return p, g, dim, A


CRIT = {"run.refine.ref_vars": "rho a1", "run.refine.rho.grad": "0.05 0.05",
        "run.refine.a1.value_range": "0.01 0.99 0.01 0.99"}


def _totals(A, dim, absolute=False):
    """Composite totals of the conserved components (masses, momenta, energy) over the uncovered
    cells of every level, weighted by the cell volume relative to level 0 (of the absolute values with
    `absolute`: the scale of a component whose total is near zero, such as the transverse momentum)."""
    cov = amr.covered_mask_fn(A.boxes, dim)
    tot = np.zeros(2 + dim + 1)
    for b, (lev, lo, hi) in enumerate(A.boxes):
        V = _valid(A.download(b), lo, hi, dim)
        m = cov(lev, lo, hi)
        for c in range(tot.size):
            v = V[c][~m]
            tot[c] += float((np.abs(v) if absolute else v).sum()) / (1 << (dim * lev))
    return tot


def test_level_tags_equal_single_box_tags():
    import torch

    p, g, dim, A = _bubble_amr()
    A.advance(3)
    crit = cb.tag_criteria(p.physics, dim, CRIT, 0, max_level=2)
    tags = A.tag(0, crit)
    # the level-0 state assembled into one box, ghosts by the physical boundary fill
    big = np.zeros(cb.padded_shape(p, g))
    ids = A.level_boxes(0)
    for b in ids:
        _, lo, hi = A.boxes[b]
        _valid(big, (0, 0, 0), (g.n[0] - 1, g.n[1] - 1, 0), dim)[:, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = \
            _valid(A.download(b), lo, hi, dim)
    Ud = torch.from_numpy(big).cuda()
    cb.FillPatch(p, g, Ud)
    t1 = torch.zeros((1, g.n[1], g.n[0]), dtype=torch.uint8, device="cuda")
    cb.tag_cells(p, g, Ud, crit, t1)
    whole = t1.cpu().numpy()[0]
    n_tagged = 0
    for b, t in zip(ids, tags):
        _, lo, hi = A.boxes[b]
        np.testing.assert_array_equal(t[0], whole[lo[1]:hi[1] + 1, lo[0]:hi[0] + 1])
        n_tagged += int(t.sum())
    A.close()
    print(f"level 0: {n_tagged} of {whole.size} cells tagged, boxes {len(ids)}")
    assert 0 < n_tagged < whole.size


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_regrid_keeps_the_state_and_the_totals(precision):
    p, g, dim, A = _bubble_amr(periodic=True, precision=precision)
    A.advance(4)
    before = {b: A.download(b) for b in range(len(A.boxes))}
    old = list(A.boxes)
    tot0 = _totals(A, dim)
    scale0 = _totals(A, dim, absolute=True)
    crit = cb.tag_criteria(p.physics, dim, CRIT, 0, max_level=2)
    new = amr.regrid_boxes([A.tag(0, crit)], old, (128, 64), dim, n_error_buf=2, blocking_factor=8,
                           max_grid_size=32)
    assert sorted(b for b in new if b[0] == 1) != sorted(b for b in old if b[0] == 1)
    A.regrid(new)
    assert A.boxes == new
    tot1 = _totals(A, dim)
    # level 0 to the bit
    for b, (lev, lo, hi) in enumerate(new):
        if lev == 0:
            ob = old.index((lev, lo, hi))
            np.testing.assert_array_equal(_valid(A.download(b), lo, hi, dim), _valid(before[ob], lo, hi, dim))
    # fine cells: copied where an old fine box held them, else children averaging to their parent
    fine_old = {}
    for ob, (lev, lo, hi) in enumerate(old):
        if lev == 1:
            V = _valid(before[ob], lo, hi, dim)
            for j in range(lo[1], hi[1] + 1):
                for i in range(lo[0], hi[0] + 1):
                    fine_old[(i, j)] = V[:, j - lo[1], i - lo[0]]
    coarse = {}
    for ob, (lev, lo, hi) in enumerate(old):
        if lev == 0:
            V = _valid(before[ob], lo, hi, dim)
            for j in range(lo[1], hi[1] + 1):
                for i in range(lo[0], hi[0] + 1):
                    coarse[(i, j)] = V[:, j - lo[1], i - lo[0]]
    n_copy = n_interp = 0
    worst = 0.0
    # per-component scale of the parent values (the transverse momentum is near zero by symmetry)
    cscale = np.maximum(np.max(np.abs(np.array(list(coarse.values()))), axis=0), 1e-300)
    for b, (lev, lo, hi) in enumerate(new):
        if lev != 1:
            continue
        V = _valid(A.download(b), lo, hi, dim)
        for j in range(lo[1], hi[1] + 1, 2):
            for i in range(lo[0], hi[0] + 1, 2):
                kids = [V[:, jj - lo[1], ii - lo[0]] for jj in (j, j + 1) for ii in (i, i + 1)]
                if (i, j) in fine_old:
                    for (ii, jj), kv in zip([(i, j), (i + 1, j), (i, j + 1), (i + 1, j + 1)],
                                            [kids[0], kids[1], kids[2], kids[3]]):
                        np.testing.assert_array_equal(kv, fine_old[(ii, jj)])
                    n_copy += 1
                else:
                    mean = (kids[0] + kids[1] + kids[2] + kids[3]) / 4.0
                    par = coarse[(i // 2, j // 2)]
                    worst = max(worst, float(np.max(np.abs(mean - par) / cscale)))
                    n_interp += 1
    rel = np.abs(tot1 - tot0) / scale0
    print(f"{precision}: regrid {sum(1 for b in old if b[0] == 1)} -> {sum(1 for b in new if b[0] == 1)} fine boxes, "
          f"{n_copy} parents copied, {n_interp} interpolated (children mean vs parent {worst:.1e}); composite totals "
          f"relative change {rel}")
    assert n_copy > 0 and n_interp > 0
    assert worst <= 1e-14
    assert np.all(rel <= 1e-14), rel
    A.advance(3)
    info = A.sync()
    assert info.status == 0 and info.steps == 7
    A.close()


def test_regrid_cycle_follows_the_interface():
    p, g, dim, A = _bubble_amr(nx=128, ny=64)
    crit = cb.tag_criteria(p.physics, dim, CRIT, 0, max_level=2)
    layouts = []
    for cycle in range(4):
        A.advance(5)
        tags = A.tag(0, crit)
        new = amr.regrid_boxes([tags], A.boxes, (128, 64), dim, n_error_buf=2, blocking_factor=8, max_grid_size=32)
        A.regrid(new)
        layouts.append(sorted(b for b in new if b[0] == 1))
        # every tagged level-0 cell at least nest cells inside the domain lies under the new fine level
        cov = amr.covered_mask_fn(new, dim)
        missed = 0
        for b, t in zip(A.level_boxes(0), tags):
            _, lo, hi = A.boxes[b]
            m = cov(0, lo, hi)
            missed += int((t[0].astype(bool) & ~m).sum())
        print(f"cycle {cycle}: {len(layouts[-1])} fine boxes, tagged cells not refined: {missed}")
        assert missed == 0
    info = A.sync()
    assert info.status == 0 and info.steps == 20
    assert len({tuple(x) for x in layouts}) > 1  # the fine level moved with the flow
    A.close()
