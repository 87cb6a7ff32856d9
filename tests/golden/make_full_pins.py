"""Pins of the configurations at their stated sizes and step counts, from the reference's OWN
arithmetic (oracle/_ref: the reference's include/Physics_* and include/Operators_* headers compiled
for the CPU). A full final state is too large to commit (256^3 x 8 fields is 1.1 GB), so a pin holds
what identifies it:

  * the SHA-256 of the initial and of the final valid cells, per field (float64, C order), and of
    every z-plane (3D) or y-row (2D) of the final state, so a mismatch names where it is;
  * the step sizes and the final time;
  * per-field sums and max |U| of the final state;
  * a sample of the final state: the centre z-plane (3D, every second cell) or every eighth cell in
    x and y (2D), for the size of a difference when the digests do not match.

The plain FP64 CUDA path reproduces the reference's arithmetic to the bit, so its test compares
digests; the sample gives the relative L-infinity on a mismatch.

Cases (run from the repository root; hours of CPU on a few cores):
  droplet_6eq_3d_128_200   3D SIXEQS shock-droplet 128^3, 200 steps (the 256^3 configuration halved)
  droplet_6eq_3d_256_200   3D SIXEQS shock-droplet 256^3, 200 steps (the configuration as stated)
  bubble_5eq_2d_2048x1024_1000  2D FIVEEQS shock-helium-bubble 2048x1024, WENO5B + HLLC, 1000 steps,
                           hyperbolic step alone (the Phase-Field step's elliptic solve is not the
                           reference's own: AMReX MLMG is not available)

  python tests/golden/make_full_pins.py droplet_6eq_3d_128_200
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import compas_b200 as cb  # noqa: E402
from compas_b200 import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
PINS = os.path.join(HERE, "pins")

CASES = {
    "droplet_6eq_3d_128_200": (cases.shock_droplet, dict(n=128), 200),
    "droplet_6eq_3d_256_200": (cases.shock_droplet, dict(n=256), 200),
    "bubble_5eq_2d_2048x1024_1000": (cases.shock_bubble, dict(nx=2048, ny=1024, scheme="WENO5B"), 1000),
}


def field_digests(V):
    """SHA-256 of each field of a valid-cell array (component-major), float64 C order."""
    return [hashlib.sha256(np.ascontiguousarray(V[c], dtype=np.float64).tobytes()).hexdigest()
            for c in range(V.shape[0])]


def plane_digests(V):
    """SHA-256 of each slowest-index slice (z-plane in 3D, y-row in 2D) over all fields."""
    W = np.ascontiguousarray(V, dtype=np.float64)
    return [hashlib.sha256(np.ascontiguousarray(W[:, k]).tobytes()).hexdigest() for k in range(W.shape[1])]


def sample(V, dim):
    """The centre z-plane at every second cell (3D) or every eighth cell in x and y (2D)."""
    if dim == 3:
        return np.ascontiguousarray(V[:, V.shape[1] // 2, ::2, ::2])
    return np.ascontiguousarray(V[:, 0, ::8, ::8])


def make(name):
    from oracle.oracle import Oracle

    fn, kw, steps = CASES[name]
    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    V0 = cb.valid_view(U, p, g)
    init = field_digests(V0)
    o = Oracle("reference", p, g)
    t0 = time.perf_counter()
    t, dts = o.advance(U, steps)
    el = time.perf_counter() - t0
    V = cb.valid_view(U, p, g)
    os.makedirs(PINS, exist_ok=True)
    np.savez_compressed(os.path.join(PINS, name + ".npz"),
                        initial_digests=np.array(init), final_digests=np.array(field_digests(V)),
                        plane_digests=np.array(plane_digests(V)), dts=dts, t=np.array([t]),
                        sums=V.reshape(V.shape[0], -1).sum(axis=1),
                        maxabs=np.abs(V).reshape(V.shape[0], -1).max(axis=1),
                        sample=sample(V, dim), inputs=np.array(repr(inputs)), geom=np.array(repr(geom)),
                        physics=np.array([phys, dim, steps]),
                        note=np.array(f"reference-header build, {o.threads()} OpenMP threads, {el:.0f} s"))
    return el


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        el = make(n)
        print("wrote", n, f"{el:.0f} s", flush=True)
