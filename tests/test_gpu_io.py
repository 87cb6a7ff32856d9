"""Plot files and checkpoints (compas_b200.io).

  * a checkpoint written after 5 steps and restarted in a new level continues the run to the bit: the
    state, the time and the step sizes after 5 more steps equal those of the uninterrupted 10 steps
    (the checkpoint keeps the last step's face wave speed, the input of the next step's ComputeDt);
  * a plot file of a level and of a multi-level hierarchy reads back to the plot variables computed
    on the device, with the header's time, step, variable names, domain and boxes.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import amr, cases, io

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case_fn,kw", [(cases.shock_droplet, dict(n=24)),
                                        (cases.shock_bubble, dict(nx=96, ny=48, scheme="WENO5B"))],
                         ids=["droplet3d", "bubble2d"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restart_continues_to_the_bit(tmp_path, case_fn, kw, precision):
    phys, dim, inputs, geom, U = case_fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": precision}))
    g = cb.make_geom(**geom)
    ref = cb.Level(p, g)
    ref.upload(U)
    ref.advance(10)
    ir = ref.sync()
    a = ref.download()
    dts_ref = ref.dts(10)
    ref.close()
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(5)
    lv.sync()
    io.write_checkpoint(str(tmp_path / "chk00005"), lv)
    lv.close()
    rs = cb.Level(p, g)
    io.read_checkpoint(str(tmp_path / "chk00005"), rs)
    rs.advance(5)
    ib = rs.sync()
    b = rs.download()
    dts = rs.dts(10)
    rs.close()
    assert ib.status == 0 and ib.steps == 10 and ib.t == ir.t
    np.testing.assert_array_equal(dts[5:], dts_ref[5:])
    np.testing.assert_array_equal(cb.valid_view(b, p, g), cb.valid_view(a, p, g))


def test_level_plotfile_reads_back(tmp_path):
    import torch

    phys, dim, inputs, geom, U = cases.shock_droplet(n=16)
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(3)
    names = ["rho", "u", "P", "a1", "T", "Mach", "vorticity_mag"]
    io.level_plotfile(str(tmp_path / "plt00003"), lv, names)
    Ud = torch.empty(cb.padded_shape(p, g), dtype=torch.float64, device="cuda")
    lv.download(out=Ud)
    info = lv.sync()
    lv.close()
    cb.FillPatch(p, g, Ud)
    out = torch.empty((len(names), 16, 16, 16), dtype=torch.float64, device="cuda")
    cb.derive(p, g, Ud, names, out)
    got_names, t, levels = io.read_plotfile(str(tmp_path / "plt00003"))
    assert got_names == names and t == info.t and len(levels) == 1
    (lo, hi, data), = levels[0]
    assert lo == (0, 0, 0) and hi == (15, 15, 15)
    np.testing.assert_array_equal(data, out.cpu().numpy())
    header = (tmp_path / "plt00003" / "Header").read_text().split("\n")
    assert header[0] == "HyperCLaw-V1.1" and header[len(names) + 2] == "3"


def test_amr_plotfile_reads_back(tmp_path):
    kw = dict(nx=64, ny=32, scheme="WENO5B")
    phys, dim, inputs, geom, _ = cases.shock_bubble(**kw, quadrature=False)
    p, g = cb.make_parm(phys, dim, inputs), cb.make_geom(**geom)
    boxes = amr.hierarchy((64, 32), dim, [((40, 16, 0), (95, 47, 0))], 16)
    A = cb.Amr(p, g, boxes)
    for b, U in enumerate(amr.box_states(cases.shock_bubble, kw, (64, 32), dim, boxes)):
        A.upload(b, U)
    A.advance(2)
    names = ["rho", "P", "a1"]
    io.amr_plotfile(str(tmp_path / "plt00002"), A, names)
    _, t, levels = io.read_plotfile(str(tmp_path / "plt00002"))
    assert len(levels) == 2
    assert sorted((lo, hi) for lo, hi, _ in levels[1]) == sorted((tuple(lo), tuple(hi)) for l, lo, hi in boxes if l == 1)
    # the plot's a1 is the state's volume fraction, box by box
    for (lev, lo, hi), b in zip([(l, tuple(lo), tuple(hi)) for l, lo, hi in boxes], range(len(boxes))):
        V = A.download(b)
        a1 = V[dim + 3, 0, 3:3 + hi[1] - lo[1] + 1, 3:3 + hi[0] - lo[0] + 1]
        data = [d for l0, h0, d in levels[lev] if l0 == lo and h0 == hi][0]
        np.testing.assert_array_equal(data[2, 0], a1)
    A.close()
