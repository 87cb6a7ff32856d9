"""The autotuner's candidates (launch shapes x tile traversal orders) of the stage kernels.

Every candidate computes the same faces with the same arithmetic, so forcing any of them must give
the same state to the bit, in the plain FP64 form and in the mixed form, for the single-box level
kernel and the box-list kernel; the tuned choice is one of the candidates."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases

pytestmark = pytest.mark.gpu

CANDIDATES = [(s, o) for s in range(3) for o in range(2)]


def _run_forced(fn, kw, precision, steps, shape, order, extra=None):
    phys, dim, inputs, geom, U = fn(**kw)
    inputs = dict(inputs, **{"compas_b200.precision": precision}, **(extra or {}))
    p, g = cb.make_parm(phys, dim, inputs), cb.make_geom(**geom)
    lv = cb.Level(p, g)
    if shape is not None:
        lv.set_kernel(shape, order)
    lv.upload(U)
    lv.advance(steps)
    info = lv.sync()
    out = lv.download()
    k = lv.kernel()
    _run_forced.tma = lv.tma()
    lv.close()
    assert info.status == 0 and info.steps == steps
    return cb.valid_view(out, p, g), k


@pytest.mark.parametrize("fn,kw,steps", [
    (cases.shock_bubble, dict(nx=72, ny=40, scheme="WENO5B"), 6),
    (cases.shock_droplet, dict(n=20), 3),
    (cases.triple_point, dict(m=8), 6),
    (cases.advected_interface, dict(n=18, dim=3, physics=cb.FIVEEQS), 3),
], ids=["bubble2d_weno5b", "droplet3d_six", "triple_nphase", "sphere3d_five"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_candidate_gives_the_same_bits(fn, kw, steps, precision):
    ref, _ = _run_forced(fn, kw, precision, steps, 0, 0)
    for shape, order in CANDIDATES[1:]:
        got, k = _run_forced(fn, kw, precision, steps, shape, order)
        assert k == (shape, order)
        assert np.array_equal(got, ref), (shape, order)
    tuned, k = _run_forced(fn, kw, precision, steps, None, None)
    print(f"autotuned choice (shape, order) = {k}")
    assert k in CANDIDATES
    assert np.array_equal(tuned, ref)


def test_batch_candidates_give_the_same_bits():
    def run(shape, order):
        b = cb.Batch(cb.FIVEEQS, 2, id_limiter=6, precision=1, capacity=8)
        if shape is not None:
            b.set_kernel(shape, order)
        ids, pgs = [], []
        for nx, ny in ((40, 24), (64, 32), (24, 24)):
            phys, dim, inputs, geom, U = cases.shock_bubble(nx=nx, ny=ny, scheme="WENO5B")
            p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
            g = cb.make_geom(**geom)
            ids.append(b.add(p, g, U, max_steps=5))
            pgs.append((p, g))
        b.advance(5)
        outs = [cb.valid_view(b.download(i), p, g) for i, (p, g) in zip(ids, pgs)]
        k = b.kernel()
        b.close()
        return outs, k

    ref, _ = run(0, 0)
    for shape, order in CANDIDATES[1:] + [(None, None)]:
        got, k = run(shape, order)
        if shape is not None:
            assert k == (shape, order)
        else:
            print(f"batch autotuned choice = {k}")
            assert k in CANDIDATES
        for a, r in zip(got, ref):
            assert np.array_equal(a, r), (shape, order)


@pytest.mark.parametrize("fn,kw,steps,uses_tma", [
    (cases.shock_droplet, dict(n=24), 4, True),
    (cases.shock_droplet, dict(n=21), 3, False),
    (cases.advected_interface, dict(n=20, dim=3, physics=cb.FIVEEQS), 3, True),
    (cases.advected_interface, dict(n=16, dim=3, physics=cb.SIXEQS), 3, True),
], ids=["droplet24", "droplet21_odd_no_tma", "sphere20_five", "sphere16_six"])
def test_tma_halo_staging_gives_the_same_bits(fn, kw, steps, uses_tma):
    """The 3D mixed form with the y/z halo slabs staged by TMA equals the plain-load form to the bit,
    for every launch shape (an odd row length falls back to plain loads)."""
    outs = {}
    for tma in (0, 1):
        for shape in range(3):
            got, k = _run_forced(fn, kw, "mixed", steps, shape, 0, {"compas_b200.tma": tma})
            assert _run_forced.tma == (bool(tma) and uses_tma)
            outs[(tma, shape)] = got
    ref = outs[(0, 0)]
    for key, got in outs.items():
        assert np.array_equal(got, ref), key
