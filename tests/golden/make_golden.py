"""Generates the golden fixtures of tests/golden from the reference's OWN arithmetic: the
reference's include/Physics_* and include/Operators_* headers compiled against the AMReX shim
(oracle/_ref, built by `make -C oracle ref` where the reference tree is present).

Each fixture holds the initial padded state, the step sizes and the valid cells after the steps,
so the CPU restatement and the CUDA path can be pinned to the reference without the reference tree.
Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import compas_b200 as cb  # noqa: E402
from compas_b200 import cases  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (case function, kwargs, steps[, extra inputs keys])
    "disc_5eq_2d_32": (cases.advected_disc, dict(n=32), 12),
    "bubble_5eq_2d_29x17": (cases.shock_bubble, dict(nx=29, ny=17, scheme="WENO5"), 6),
    "droplet_6eq_3d_12": (cases.shock_droplet, dict(n=12), 3),
    "bubble_weno5b_5eq_2d_31x19": (cases.shock_bubble, dict(nx=31, ny=19, scheme="WENO5B"), 6),
    "disc_thinc_5eq_2d_32": (cases.advected_disc, dict(n=32), 12, {"FiniteVolume.THINC": "1"}),
    "bubble_thinc_weno5b_5eq_2d_31x19": (cases.shock_bubble, dict(nx=31, ny=19, scheme="WENO5B"), 6,
                                         {"FiniteVolume.THINC": "1", "FiniteVolume.THINC.UseNormal": "0"}),
    "droplet_thinc_6eq_3d_12": (cases.shock_droplet, dict(n=12), 3, {"FiniteVolume.THINC": "1"}),
    "triple_5eqn3_2d_42x18": (cases.triple_point, dict(m=6), 10),
    "bubbles_nasg_k_5eqn4_2d_24": (cases.nphase_bubbles, dict(n=24, nphase=4, eos=3, source_term=1), 6),
    "bubbles_5eqn2_2d_24": (cases.nphase_bubbles, dict(n=24, nphase=2), 6),
    "bubbles_5eqn3_3d_10": (cases.nphase_bubbles, dict(n=10, nphase=3, dim=3), 3),
    "shockbubble_6eqn2_2d_24x12": (cases.sixn_shock_bubbles, dict(n=12, nphase=2, dp=0.05), 6),
    "shockbubbles_nasg_6eqn3_2d_32x16": (cases.sixn_shock_bubbles, dict(n=16, nphase=3, eos=3, dp=0.05,
                                                                       scheme="WENO5B"), 6),
    "shockbubbles_6eqn3_3d_16x8x8": (cases.sixn_shock_bubbles, dict(n=8, nphase=3, dim=3, dp=0.05), 3),
}


def make(name):
    fn, kw, steps = CASES[name][:3]
    phys, dim, inputs, geom, U = fn(**kw)
    inputs = dict(inputs, **(CASES[name][3] if len(CASES[name]) > 3 else {}))
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    out = U.copy()
    t, dts = Oracle("reference", p, g).advance(out, steps)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), U0=U, dts=dts, t=np.array([t]),
                        valid=np.ascontiguousarray(cb.valid_view(out, p, g)),
                        inputs=np.array(repr(inputs)), geom=np.array(repr(geom)),
                        physics=np.array([phys, dim, steps]))


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        make(n)
        print("wrote", n)
