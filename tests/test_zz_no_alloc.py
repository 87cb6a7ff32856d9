"""The allocation-free RK3 step (compas_b200_rk3_step_noalloc), for callers that cannot allocate device
memory themselves or through the library - when another allocator (an AMReX arena, a framework's
caching allocator) must stay the only owner of device memory, or the reservation is fixed. It keeps the two intermediate stage states in the
library's fixed device scratch array, so it is checked here against the existing entry points, which
take those states from the caller: boundary fill + compas_b200_rk3_stage, three times per step, with
caller-allocated stage buffers. Two steps in a row, both must agree to the bit (the same kernels run
on the same data; the parity tolerance of the FP64 tests is 1e-11 relative). This file is collected
last so that a failure here cannot stop the other tests."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases

pytestmark = pytest.mark.gpu


def _reference_step(torch, p, g, U, dt):
    """One step through the existing per-stage entry points with caller-owned stage buffers."""
    U1 = torch.zeros_like(U)
    U2 = torch.zeros_like(U)
    dt_dev = torch.tensor([dt], dtype=torch.float64, device="cuda")
    ins, outs = (U, U1, U2), (U1, U2, U)
    for s in range(3):
        cb.FillPatch(p, g, ins[s])
        cb.ThirdOrderSSPRK_stage(p, g, s, ins[s], U, outs[s], dt_dev)


@pytest.mark.parametrize("case,kw,precision", [
    (cases.advected_disc, dict(n=64), "fp64"),
    (cases.shock_droplet, dict(n=24), "fp64"),
    (cases.shock_bubble, dict(nx=96, ny=48, scheme="WENO5B"), "mixed"),
])
def test_noalloc_step_matches_stage_entry_points_twice(case, kw, precision):
    import torch

    phys, dim, inputs, geom, U0 = case(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": precision}))
    g = cb.make_geom(**geom)
    a = torch.from_numpy(U0).cuda()
    b = a.clone()
    cm_a = torch.zeros(1, dtype=torch.float64, device="cuda")
    cm_b = torch.zeros(1, dtype=torch.float64, device="cuda")
    cb.FillPatch(p, g, a)
    cb.compute_dUdt_FV(p, g, a, torch.zeros_like(a), cmax=cm_a)
    torch.cuda.synchronize()
    dt = 0.4 * min(g.dx[0], g.dx[1]) / float(cm_a.item())
    for call in range(2):
        cb.ThirdOrderSSPRK_step_noalloc(p, g, a, dt, cmax=cm_a)
        _reference_step(torch, p, g, b, dt)
        torch.cuda.synchronize()
        va = cb.valid_view(a.cpu().numpy(), p, g)
        vb = cb.valid_view(b.cpu().numpy(), p, g)
        assert np.isfinite(va).all()
        np.testing.assert_array_equal(va, vb, err_msg=f"call {call}")


def test_noalloc_step_rejects_states_beyond_its_scratch():
    phys, dim, inputs, geom, _ = cases.advected_disc(n=8, quadrature=False)
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom((1024, 1024, 1), (1.0 / 1024, 1.0 / 1024, 1.0), 3, (0, 0, 0), (0, 0, 0))
    assert cb.lib().compas_b200_state_bytes(p, g) > 16 << 20
    with pytest.raises(cb.CompasError) as e:
        cb.ThirdOrderSSPRK_step_noalloc(p, g, 0x1000, 1e-6)  # rejected before any device access
    assert e.value.code == cb.EARG
