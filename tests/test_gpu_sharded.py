"""The sharded single-level advance on one GPU: the case cut into 2 or 3 slabs held in one process
(LocalComm: ghost planes copied between the slabs' arrays), each slab advanced through the C ABI's
boundary fill and fused stage entry points. The slabs together must give the single-box level advance
to the bit, state and every step size, in both precision forms."""
import numpy as np
import pytest
import torch

import compas_b200 as cb
from compas_b200 import cases, sharded

pytestmark = pytest.mark.gpu


def _run_level(p, g, U, steps):
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(steps, use_graph=False)
    info = lv.sync()
    out = cb.valid_view(lv.download(), p, g)
    dts = lv.dts(info.steps)
    lv.close()
    return out, dts, info


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case,kw,world,steps", [
    (cases.shock_droplet, dict(n=32), 2, 4),
    (cases.shock_droplet, dict(n=30), 3, 3),
    (cases.advected_disc, dict(n=64), 2, 5),
    (cases.advected_disc, dict(n=48), 3, 5),
])
def test_slabs_match_single_box_level(precision, case, kw, world, steps):
    assert torch.cuda.is_available()
    phys, dim, inputs, geom, U = case(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": precision}))
    g = cb.make_geom(**geom)
    want, dts_want, info = _run_level(p, g, U, steps)
    assert info.status == 0 and info.steps == steps
    sl = sharded.ShardedLevel(p, g, sharded.LocalComm(world))
    sl.upload(U)
    assert sl.advance(steps) == steps
    torch.cuda.synchronize()
    assert sl.status() == 0
    got = np.zeros_like(want)
    for idx, v in sl.download():
        got[idx] = v.cpu().numpy()
    np.testing.assert_array_equal(np.array(sl.dts), dts_want)
    np.testing.assert_array_equal(got, want)
