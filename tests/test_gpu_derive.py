"""Plot variables on the device (compas_b200_derive) against the reference's own compute_derived_var
(ComputeDerivedVar_Compressible5Eq.H / _Compressible6Eq.H with DerivedVelocityGradient.H), compiled in
the oracle: every state and derived variable of the two-phase models on the shock-bubble and the
shock-droplet after some steps, cell for cell. The derived values are the reference's formulas in its
order of operations, so they are equal to the bit, except lambda2, whose closed-form eigenvalues call
acos and cos (CUDA's and the host library's may differ in the last bit): it is held to 1e-12 relative
to its largest magnitude."""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import oracle_kind
from oracle.oracle import Oracle, have_ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,case_fn,kw,steps,cv", [
    ("bubble2d", cases.shock_bubble, dict(nx=96, ny=48, scheme="WENO5B"), 40, ("0.717", "3.12")),
    ("droplet3d", cases.shock_droplet, dict(n=24), 10, ("717.5", "4180.0")),
], ids=["bubble2d", "droplet3d"])
def test_derived_variables_equal_the_reference(name, case_fn, kw, steps, cv):
    import torch

    phys, dim, inputs, geom, U = case_fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"prob.EOS.cv_1": cv[0], "prob.EOS.cv_2": cv[1]}))
    g = cb.make_geom(**geom)
    if not have_ref(p.physics, p.dim):
        pytest.skip("reference-header oracle not built")
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(steps)
    Ud = torch.empty(cb.padded_shape(p, g), dtype=torch.float64, device="cuda")
    lv.download(out=Ud)
    lv.close()
    cb.FillPatch(p, g, Ud)
    names = cb._DERIVED_NAMES[p.physics]
    nz = g.n[2] if dim == 3 else 1
    out = torch.zeros((len(names), nz, g.n[1], g.n[0]), dtype=torch.float64, device="cuda")
    cb.derive(p, g, Ud, names, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    o = Oracle(oracle_kind(p.physics, p.dim), p, g)
    ref = o.derive(Ud.cpu().numpy(), [cb.tag_variable(p.physics, dim, nm) for nm in names], cv=(p.cv_1, p.cv_2))
    for v, nm in enumerate(names):
        if nm == "lambda2":
            scale = max(float(np.abs(ref[v]).max()), 1e-300)
            e = float(np.abs(got[v] - ref[v]).max()) / scale
            print(f"{name} {nm}: max relative difference {e:.1e}")
            assert e <= 1e-12, (nm, e)
        else:
            np.testing.assert_array_equal(got[v], ref[v], err_msg=nm)
    print(f"{name}: {len(names)} variables equal to the reference's compute_derived_var")
