"""Refinement tagging on the device (compas_b200_tag_cells) against the reference's own ErrorEst tests:
the oracle compiles include/Tagging.H (state_grad, state_value_less / greater / range) and the
models' compute_derived_var (ComputeDerivedVar_Compressible5Eq.H / _Compressible6Eq.H, with the
velocity-gradient invariants of DerivedVelocityGradient.H) and tags the same ghost-filled state. The
tag sets must be equal, cell for cell, on the shock-bubble and the shock-droplet after some steps
(shocks, interfaces and vorticity present), for criteria on state and derived variables of every
kind, the thresholds read from run.refine.* keys as the reference reads them."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import oracle_kind
from oracle.oracle import Oracle, have_ref

pytestmark = pytest.mark.gpu

INPUTS_5EQ = {
    "run.refine.ref_vars": "rho a1 P vorticity_mag Mach T rho_E q_criterion lambda2 u",
    "run.refine.rho.grad": "0.1 0.2",
    "run.refine.a1.value_range": "0.01 0.99 0.05 0.95",
    "run.refine.P.value_greater": "1.3 1.6",
    "run.refine.vorticity_mag.grad": "0.01 0.05",
    "run.refine.Mach.value_greater": "0.1 0.3",
    "run.refine.T.grad": "0.01 0.05",
    "run.refine.rho_E.grad": "0.1 0.2",
    "run.refine.q_criterion.value_less": "-1e-3 -1e-2",
    "run.refine.lambda2.value_greater": "1e-7 1e-6",
    "run.refine.u.value_greater": "0.01 0.1",
    "run.refine.u.max_level": "1",
    "prob.EOS.cv_1": "0.717", "prob.EOS.cv_2": "3.12",
}
INPUTS_6EQ = {
    "run.refine.ref_vars": "a1 rho a2P2 a1P1 P vorticity_mag T c",
    "run.refine.a1.value_range": "0.001 0.999 0.01 0.99",
    "run.refine.rho.grad": "10.0 50.0",
    "run.refine.a2P2.value_greater": "1e3 1e4",
    "run.refine.a1P1.grad": "1e4 5e4",
    "run.refine.P.value_less": "1.0e5 9.99e4",
    "run.refine.vorticity_mag.grad": "100.0 500.0",
    "run.refine.T.grad": "10.0 50.0",
    "run.refine.c.grad": "30.0 100.0",
    "prob.EOS.cv_1": "717.5", "prob.EOS.cv_2": "4180.0",
}


def _state(case_fn, kw, steps, inputs_extra):
    phys, dim, inputs, geom, U = case_fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **inputs_extra))
    g = cb.make_geom(**geom)
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(steps)
    out = lv.download()
    lv.close()
    return p, g, out, dict(inputs, **inputs_extra)


@pytest.mark.parametrize("name,case_fn,kw,steps,tag_inputs", [
    ("bubble2d", cases.shock_bubble, dict(nx=160, ny=80, scheme="WENO5B"), 60, INPUTS_5EQ),
    ("droplet3d", cases.shock_droplet, dict(n=32), 12, INPUTS_6EQ),
], ids=["bubble2d", "droplet3d"])
def test_tags_equal_the_reference_errorest(name, case_fn, kw, steps, tag_inputs):
    import torch

    p, g, U, inputs = _state(case_fn, kw, steps, {k: v for k, v in tag_inputs.items() if k.startswith("prob.")})
    if not have_ref(p.physics, p.dim):
        pytest.skip("reference-header oracle not built")
    Ud = torch.from_numpy(U).cuda()
    cb.FillPatch(p, g, Ud)
    Uf = Ud.cpu().numpy()
    o = Oracle(oracle_kind(p.physics, p.dim), p, g)
    nz = g.n[2] if p.dim == 3 else 1
    for lev in (0, 1):
        crit = cb.tag_criteria(p.physics, p.dim, tag_inputs, lev, max_level=2)
        assert crit, "no criteria"
        tags = torch.zeros((nz, g.n[1], g.n[0]), dtype=torch.uint8, device="cuda")
        cb.tag_cells(p, g, Ud, crit, tags)
        torch.cuda.synchronize()
        got = tags.cpu().numpy()
        ref = o.tag(Uf, [(c.var, c.derived, c.kind, c.v0, c.v1) for c in crit], cv=(p.cv_1, p.cv_2))
        # each criterion on its own too, so that a mismatch names its variable
        per = []
        for c in crit:
            t1 = torch.zeros_like(tags)
            cb.tag_cells(p, g, Ud, [c], t1)
            torch.cuda.synchronize()
            r1 = o.tag(Uf, [(c.var, c.derived, c.kind, c.v0, c.v1)], cv=(p.cv_1, p.cv_2))
            per.append((c.var, c.derived, c.kind, int(r1.sum()), int((t1.cpu().numpy() != r1).sum())))
        print(f"{name} level {lev}: {len(crit)} criteria, {int(ref.sum())} of {ref.size} cells tagged; "
              f"per criterion (var, derived, kind, tagged, mismatches): {per}")
        assert 0 < int(ref.sum()) < ref.size
        assert all(m == 0 for *_, m in per), per
        np.testing.assert_array_equal(got, ref)


def test_tagging_rejects_bad_criteria():
    import torch

    phys, dim, inputs, geom, U = cases.advected_disc(n=16)
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    Ud = torch.from_numpy(U).cuda()
    tags = torch.zeros((1, 16, 16), dtype=torch.uint8, device="cuda")
    with pytest.raises(cb.CompasError):
        cb.tag_cells(p, g, Ud, [cb.TagCriterion(40, 1, cb.TAG_GRAD, 1.0, 0.0)], tags)
    with pytest.raises(cb.CompasError):
        cb.tag_cells(p, g, Ud, [cb.TagCriterion(0, 0, 9, 1.0, 0.0)], tags)
    with pytest.raises(cb.CompasError):
        cb.tag_cells(p, g, Ud, [cb.TagCriterion(0, 0, cb.TAG_LESS, 1.0, 0.0)] * 17, tags)
