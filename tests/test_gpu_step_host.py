"""The host-buffer step (compas_b200_level_step_host): the state moves in and out in slabs of tile layers,
the copies overlapped with the stages of neighbouring slabs. It runs the level's kernels on the same tiles,
so every step must equal set_state + advance(1) + download to the bit: checked over consecutive steps, the
output of one step fed back as the input of the next, for several slab counts, both precisions, 3D slabs
along z and 2D slabs along y (reflecting walls there), and the fallback of a periodic slab direction."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    assert torch.cuda.is_available()
    return torch


CASES = [
    (cases.shock_droplet, dict(n=40), "mixed", 2),
    (cases.shock_droplet, dict(n=40), "mixed", 3),
    (cases.shock_droplet, dict(n=40), "fp64", 64),
    (cases.shock_bubble, dict(nx=96, ny=80, scheme="WENO5B"), "mixed", 4),
    (cases.shock_bubble, dict(nx=96, ny=80, scheme="WENO5B"), "fp64", 2),
    (cases.advected_interface, dict(n=24, dim=3, physics=cb.SIXEQS), "mixed", 3),
]
IDS = ["droplet3d_mixed_2", "droplet3d_mixed_3", "droplet3d_fp64_64", "bubble2d_mixed_4", "bubble2d_fp64_2",
       "periodic3d_fallback"]


@pytest.mark.parametrize("fn,kw,prec,slabs", CASES, ids=IDS)
def test_step_host_equals_set_state_advance_download(fn, kw, prec, slabs):
    torch = _torch()
    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec}))
    g = cb.make_geom(**geom)
    ref, new = cb.Level(p, g), cb.Level(p, g)
    ref.upload(U)
    new.upload(U)
    shape = cb.padded_shape(p, g)
    a_in = torch.from_numpy(U.copy()).pin_memory()
    b_in = torch.from_numpy(U.copy()).pin_memory()
    a_out = torch.empty(shape, dtype=torch.float64).pin_memory()
    b_out = torch.empty(shape, dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream()
    for step in range(4):
        ref.set_state(a_in, stream=stream)
        ref.advance(1, stream=stream)
        ref.download(out=a_out, stream=stream)
        new.step_host(b_in, b_out, slabs=slabs, stream=stream)
        torch.cuda.synchronize()
        A, B = a_out.numpy(), b_out.numpy()
        assert np.array_equal(cb.valid_view(A, p, g), cb.valid_view(B, p, g)), step
        a_in.copy_(a_out)
        b_in.copy_(b_out)
    ia, ib = ref.sync(), new.sync()
    assert ia.status == 0 and ib.status == 0 and ia.steps == ib.steps == 4
    np.testing.assert_array_equal(ref.dts(4), new.dts(4))
    ref.close()
    new.close()


def test_step_host_in_place():
    """host_in and host_out may be the same array."""
    torch = _torch()
    phys, dim, inputs, geom, U = cases.shock_droplet(n=32)
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    g = cb.make_geom(**geom)
    ref, new = cb.Level(p, g), cb.Level(p, g)
    ref.upload(U)
    new.upload(U)
    h = torch.from_numpy(U.copy()).pin_memory()
    for _ in range(3):
        ref.advance(1)
        new.step_host(h, h, slabs=4)
    torch.cuda.synchronize()
    assert np.array_equal(cb.valid_view(ref.download(), p, g), cb.valid_view(h.numpy(), p, g))
    ref.close()
    new.close()
