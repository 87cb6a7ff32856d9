"""The batched form: many independent cases of uneven size in one persistent box-list launch per RK
stage. Each case's result must be the same alone (a single-case level) and in the mix, to the bit,
in both precision forms; admitting and retiring cases between CUDA-graph replays must not disturb the
others; a case stops at its own step budget."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import run_gpu

pytestmark = pytest.mark.gpu


def _bubbles(precision, scheme="WENO5B"):
    rng = np.random.default_rng(0)
    out = []
    for nx, ny in ((48, 32), (64, 64), (37, 23), (96, 48), (16, 16)):
        Ma = float(rng.uniform(1.1, 3.0))
        rb = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
        phys, dim, inputs, geom, U = cases.shock_bubble(nx=nx, ny=ny, Ma=Ma, rho_b=rb, scheme=scheme,
                                                        radius=float(rng.uniform(0.1, 0.3)))
        inputs = dict(inputs, **{"compas_b200.precision": precision})
        out.append((cb.make_parm(phys, dim, inputs), cb.make_geom(**geom), U))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_alone_fiveeq_2d(precision):
    cs = _bubbles(precision)
    prec = 1 if precision == "mixed" else 0
    b = cb.Batch(cb.FIVEEQS, 2, id_limiter=6, precision=prec)
    ids = [b.add(p, g, U) for p, g, U in cs]
    b.advance(8)
    infos = {i.id: i for i in b.poll()}
    for cid, (p, g, U) in zip(ids, cs):
        alone, info, _ = run_gpu(p, g, U, 8)
        got = b.download(cid)
        assert infos[cid].steps == 8 and infos[cid].status == 0
        assert infos[cid].t == info.t
        np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(alone, p, g))
    b.close()


def test_batch_step_budget_and_admission_between_replays():
    cs = _bubbles("fp64", scheme="WENO5")
    b = cb.Batch(cb.FIVEEQS, 2, id_limiter=5)
    a = b.add(*cs[0], max_steps=3)
    c = b.add(*cs[1])
    b.advance(5)                       # graph captured here
    d = b.add(*cs[2])                  # admitted between replays
    b.remove(c)                        # retired between replays
    b.advance(4)
    infos = {i.id: i for i in b.poll()}
    assert infos[a].steps == 3 and infos[a].done
    assert infos[d].steps == 4
    ref_a, _, _ = run_gpu(*cs[0], 3)
    ref_d, _, _ = run_gpu(*cs[2], 4)
    np.testing.assert_array_equal(cb.valid_view(b.download(a), cs[0][0], cs[0][1]), cb.valid_view(ref_a, cs[0][0], cs[0][1]))
    np.testing.assert_array_equal(cb.valid_view(b.download(d), cs[2][0], cs[2][1]), cb.valid_view(ref_d, cs[2][0], cs[2][1]))
    b.close()


def test_batch_sixeq_3d_two_sizes():
    out = []
    for n in (16, 24):
        phys, dim, inputs, geom, U = cases.shock_droplet(n=n)
        out.append((cb.make_parm(phys, dim, inputs), cb.make_geom(**geom), U))
    b = cb.Batch(cb.SIXEQS, 3)
    ids = [b.add(p, g, U) for p, g, U in out]
    b.advance(3)
    for cid, (p, g, U) in zip(ids, out):
        alone, _, _ = run_gpu(p, g, U, 3)
        np.testing.assert_array_equal(cb.valid_view(b.download(cid), p, g), cb.valid_view(alone, p, g))
    b.close()


def test_serving_results_identical_alone_and_in_the_mix():
    """Continuous batching: requests admitted while others run give the same state as alone."""
    from compas_b200 import serving

    reqs = serving.poisson_requests(9, rate=200.0, seed=1, sides2d=(32, 64), sides3d=(16, 24), sides_triple=(16, 32),
                                    steps=(5, 12))
    assert {r.kind for r in reqs} == set(serving.KINDS)
    srv = serving.Server(budget_bytes=150e9, precision="mixed", keep_results=True, steps_per_iter=1)
    done = srv.run(reqs)
    srv.close()
    assert len(done) == len(reqs)
    overlap = sum(1 for a in done for b in done if a is not b and a.admitted < b.finished and b.admitted < a.finished)
    assert overlap > 0, "no request overlapped another"
    for r in done:
        p, g, U = serving.make_case(r, "mixed")
        alone, info, _ = run_gpu(p, g, U.cpu().numpy(), r.steps)
        assert info.steps == r.steps
        np.testing.assert_array_equal(cb.valid_view(r.result, p, g), cb.valid_view(alone, p, g))


def test_serving_budget_admission_waits():
    from compas_b200 import serving

    reqs = serving.poisson_requests(4, rate=1000.0, seed=2, kinds=("bubble2d",), sides2d=(64, 64), steps=(4, 4))
    one = 3 * 6 * (64 + 6) * (64 + 6) * 8
    srv = serving.Server(budget_bytes=one * 1.5, precision="fp64", steps_per_iter=1)
    done = srv.run(reqs)
    srv.close()
    # with room for one case at a time, no two requests overlap
    spans = sorted((r.admitted, r.finished) for r in done)
    assert all(spans[i][1] <= spans[i + 1][0] + 1e-9 for i in range(len(spans) - 1))
