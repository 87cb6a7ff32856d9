"""Parity of the plain FP64 path with the reference's own arithmetic at the configurations' stated sizes
and step counts, against the pins of tests/golden/pins (made by tests/golden/make_full_pins.py from
the reference-header CPU build: digests of every field, the step sizes, sums, and a sample).

The FP64 path reproduces the reference's arithmetic to the bit, so a pin is met when the SHA-256 of
every field of the final state and every step size are equal; this is stronger than the 1e-11
relative L-infinity bound, which is what a mismatch is then measured against on the pin's sample.
The initial state is rebuilt here by the same numpy case builder and checked against the pin's
initial digests first, so a host whose math library rounds differently is reported as such.
"""
import hashlib
import os

import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases

pytestmark = pytest.mark.gpu

PINS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pins")
BUILDERS = {
    "droplet_6eq_3d_128_200": (cases.shock_droplet, dict(n=128)),
    "droplet_6eq_3d_256_200": (cases.shock_droplet, dict(n=256)),
    "bubble_5eq_2d_2048x1024_1000": (cases.shock_bubble, dict(nx=2048, ny=1024, scheme="WENO5B")),
}
TOL = 1e-11


def _digests(V):
    return [hashlib.sha256(np.ascontiguousarray(V[c], dtype=np.float64).tobytes()).hexdigest()
            for c in range(V.shape[0])]


def _plane_digests(V):
    W = np.ascontiguousarray(V, dtype=np.float64)
    return [hashlib.sha256(np.ascontiguousarray(W[:, k]).tobytes()).hexdigest() for k in range(W.shape[1])]


def _sample(V, dim):
    if dim == 3:
        return np.ascontiguousarray(V[:, V.shape[1] // 2, ::2, ::2])
    return np.ascontiguousarray(V[:, 0, ::8, ::8])


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_fp64_matches_the_reference_at_the_stated_size(name):
    path = os.path.join(PINS, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"pin {name} not generated (tests/golden/make_full_pins.py)")
    pin = np.load(path)
    fn, kw = BUILDERS[name]
    phys, dim, inputs, geom, U = fn(**kw)
    steps = int(pin["physics"][2])
    assert repr(inputs) == str(pin["inputs"]) and repr(geom) == str(pin["geom"])
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    init = _digests(cb.valid_view(U, p, g))
    assert init == list(pin["initial_digests"]), \
        "the numpy case builder gives a different initial state on this host (math-library rounding)"
    lv = cb.Level(p, g)
    lv.upload(U)
    del U
    lv.advance(steps, use_graph=True)
    info = lv.sync()
    dts = lv.dts(info.steps)
    out = lv.download()
    lv.close()
    V = cb.valid_view(out, p, g)
    assert info.status == 0 and info.steps == steps
    np.testing.assert_array_equal(dts, pin["dts"])
    assert info.t == float(pin["t"][0])
    got = _digests(V)
    sums = V.reshape(V.shape[0], -1).sum(axis=1)
    sample = _sample(V, dim)
    ref_sample = pin["sample"]
    den = np.maximum(np.abs(ref_sample).reshape(ref_sample.shape[0], -1).max(axis=1), 1e-300)
    e = np.abs(sample - ref_sample).reshape(sample.shape[0], -1).max(axis=1) / den
    same = [a == b for a, b in zip(got, pin["final_digests"])]
    bad_planes = [k for k, (a, b) in enumerate(zip(_plane_digests(V), pin["plane_digests"])) if a != b]
    print(f"{name}: {steps} steps, dt sequence equal, fields bit-identical {same}, "
          f"sample rel Linf {e}, planes differing {len(bad_planes)}")
    assert np.all(e <= TOL), (e, bad_planes[:10])
    assert all(same), (same, bad_planes[:10])
    np.testing.assert_allclose(sums, pin["sums"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("scheme", ["WENO5", "WENO5B"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shock_droplet_conserves_on_a_periodic_box(precision, scheme):
    """The shock-droplet of the 3D configuration (64^3, 200 steps) with periodic boundaries: the masses,
    the momenta and the total energy (the sum of the two phase energies) are conserved to round-off in
    both precision forms; with the bounded scheme (WENO5B) the volume fraction stays in [0, 1]."""
    phys, dim, inputs, geom, U = cases.shock_droplet(n=64)
    geom = dict(geom, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": precision, "FiniteVolume.Scheme": scheme}))
    g = cb.make_geom(**geom)

    def totals(V):
        return np.array([V[0].sum(), V[1].sum(), V[2].sum(), V[3].sum(), V[4].sum(), V[5].sum() + V[6].sum()])

    V0 = cb.valid_view(U, p, g)
    mom = sum(np.abs(V0[c]).sum() for c in (2, 3, 4))
    scale = np.array([np.abs(V0[0]).sum(), np.abs(V0[1]).sum(), mom, mom, mom,
                      np.abs(V0[5]).sum() + np.abs(V0[6]).sum()])
    tot0 = totals(V0)
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(200, use_graph=True)
    info = lv.sync()
    V = cb.valid_view(lv.download(), p, g)
    lv.close()
    assert info.status == 0 and info.steps == 200
    err = np.abs(totals(V) - tot0) / scale
    print(f"{precision} {scheme}: periodic shock-droplet 64^3 x 200 steps, relative change of the masses, "
          f"momenta, total energy: {err}; alpha1 in [{V[7].min():.3e}, {V[7].max():.3e}]")
    # the mixed relaxation keeps the entry momentum and total energy of a cell to the bit (the larger
    # phase takes the remainder of the total), so both forms conserve the total energy to round-off
    assert np.all(err <= 1e-13), err
    if scheme == "WENO5B":
        assert V[7].min() >= 0.0 and V[7].max() <= 1.0
