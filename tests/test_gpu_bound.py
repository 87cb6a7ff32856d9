"""Bound-preserving path of the five-equation model (FiniteVolume.ID_Bound = 1) against the reference's
own headers compiled in the oracle:

  * the right-hand side (compas_b200_compute_dUdt): MUSCLBP for GODUNOV and every MUSCL limiter,
    WENO5BP for WENO3 / WENO3B (quadrature weight 1/6) and WENO5 / WENO5B (1/12), the energy-bound
    limiter, the HLL solver with bounded wave speeds under both ID_Lambda values, the CFL speed of the
    branch, with and without the Kapila term, on the shock-bubble and on a stressed state (near-zero
    pressure of the air, large velocity jumps) where the limiter and the general speed bound act:
    equal to the bit, and the wave speed too;
  * the face fluxes of that branch (compas_b200_face_fluxes): their divergence is the right-hand side;
  * MinEnergyBound (compas_b200_energy_bound_min) to the bit;
  * the level advance with its energy check after every stage and the step taken again with the
    general bound when a stage violates it (source/Class_Compressible_PhaseField.cpp:236-306):
    state, dt sequence and the number of restarts equal to the reference's loop, in a run that
    restarts.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from compas_b200.cases import _cons_from_prims
from oracle.oracle import Oracle, have_ref

pytestmark = pytest.mark.gpu

SCHEMES = ["GODUNOV", "MUSCL", "MUSCL-vanLeer", "MUSCL-Superbee", "MUSCL-MC", "WENO3", "WENO3B", "WENO5",
           "WENO5B"]


def _bubble(scheme, extra=None, nx=48, ny=24):
    phys, dim, inputs, geom, U = cases.shock_bubble(nx=nx, ny=ny, scheme="WENO5", quadrature=False)
    inp = dict(inputs, **{"FiniteVolume.Scheme": scheme, "FiniteVolume.ID_Bound": 1}, **(extra or {}))
    return cb.make_parm(phys, dim, inp), cb.make_geom(**geom), U


STATES = {
    # air (gamma 1.4) and helium (gamma 1.648), pressures 1e-4..1e-1 (the air's p_min is 0), velocities
    # +-50: the cells' energy bound is small against their kinetic energy, so reconstructed and
    # quadrature states violate it and the energy-bound limiter acts
    "air_helium_low_p": dict(gamma2=1.648, pinf2=0.0, rho2=(0.1, 0.3), logp=(-4.0, -1.0), source_term=0),
    # air and water (stiffened gas gamma 4.4, p_inf 6e8) with the Kapila term: in mixed cells the
    # general wave-speed bound of ID_Lambda = 0 departs from the sound speed
    "air_water_kapila": dict(gamma2=4.4, pinf2=6e8, rho2=(900.0, 1100.0), logp=(3.0, 6.0), source_term=1),
}


def _stressed_case(dim, scheme, state, seed=7):
    """A padded five-equation state of random cells (volume fractions in [0, 1] with pure cells,
    velocities of +-50, the pressures and second phase of STATES[state])."""
    s = STATES[state]
    phys, _, inputs, geom, _ = cases.shock_bubble(nx=40, ny=24, scheme="WENO5", quadrature=False)
    if dim == 3:
        geom = dict(n=(16, 12, 10), dx=(0.05, 0.05, 0.05), ng=3, lo_bc=(2, 4, 0), hi_bc=(2, 4, 0))
    inp = dict(inputs, **{"FiniteVolume.Scheme": scheme, "FiniteVolume.ID_Bound": 1, "prob.EOS.gamma_2": s["gamma2"],
                          "prob.EOS.pinf_2": s["pinf2"], "Physics.source_term": s["source_term"]})
    p = cb.make_parm(phys, dim, inp)
    g = cb.make_geom(**geom)
    rng = np.random.Generator(np.random.PCG64(seed + dim))
    shp = cb.padded_shape(p, g)[1:]
    a1 = np.clip(rng.uniform(-0.3, 1.3, shp), 0.0, 1.0)
    r1 = rng.uniform(0.5, 2.0, shp)
    r2 = rng.uniform(*s["rho2"], shp)
    vel = [rng.uniform(-50.0, 50.0, shp) for _ in range(dim)]
    pr = 10.0 ** rng.uniform(*s["logp"], shp)
    g2 = s["gamma2"]
    A = (1.0 / 0.4, 1.0 / (g2 - 1.0))
    B = (0.0, g2 * s["pinf2"] / (g2 - 1.0))
    U = _cons_from_prims(p.physics, dim, a1 * r1, (1.0 - a1) * r2, vel, pr, a1, A, B, np)
    return p, g, np.ascontiguousarray(U)


def _dudt_pair(p, g, U):
    import torch

    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    Ud = torch.from_numpy(U.copy()).cuda()
    cb.FillPatch(p, g, Ud)
    dU = torch.zeros_like(Ud)
    cmax = torch.zeros(1, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    cb.compute_dUdt_FV(p, g, Ud, dU, cmax, err)
    torch.cuda.synchronize()
    Uf = Ud.cpu().numpy()
    o = Oracle("reference", p, g)
    ref, cm_ref = o.compute_dudt(Uf)
    return cb.valid_view(dU.cpu().numpy(), p, g), cb.valid_view(ref, p, g), float(cmax.item()), cm_ref, Uf


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("source_term", [0, 1])
def test_rhs_shock_bubble_equals_the_reference(scheme, source_term):
    p, g, U = _bubble(scheme, {"Physics.source_term": source_term})
    got, ref, cm, cm_ref, _ = _dudt_pair(p, g, U)
    np.testing.assert_array_equal(got, ref)
    assert cm == cm_ref, (cm, cm_ref)


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("id_lambda", [1, 0])
@pytest.mark.parametrize("state", list(STATES))
def test_rhs_stressed_state_equals_the_reference(scheme, dim, id_lambda, state):
    p, g, U = _stressed_case(dim, scheme, state)
    p.id_lambda = id_lambda
    got, ref, cm, cm_ref, _ = _dudt_pair(p, g, U)
    np.testing.assert_array_equal(got, ref)
    assert cm == cm_ref, (cm, cm_ref)


def test_general_bound_changes_the_speeds():
    """On the air-water state with the Kapila term the general bound (ID_Lambda = 0) gives other wave
    speeds and fluxes than the sound speed: the branch under test is not the ID_Lambda = 1 one."""
    p, g, U = _stressed_case(2, "MUSCL", "air_water_kapila")
    got1, _, cm1, _, _ = _dudt_pair(p, g, U)
    p.id_lambda = 0
    got0, _, cm0, _, _ = _dudt_pair(p, g, U)
    print(f"cmax: ID_Lambda 1 {cm1:.6e}, ID_Lambda 0 {cm0:.6e}")
    assert cm0 > cm1 and not np.array_equal(got0, got1)


@pytest.mark.parametrize("scheme", ["MUSCL-MC", "WENO5B"])
def test_face_flux_divergence_is_the_rhs(scheme):
    import torch

    p, g, U = _stressed_case(2, scheme, "air_helium_low_p")
    got, _, _, _, Uf = _dudt_pair(p, g, U)
    N = cb.parm_nstate(p)
    F = [torch.zeros(cb.face_shape(p, g, d, N), dtype=torch.float64, device="cuda") for d in range(2)]
    Fn = [torch.zeros(cb.face_shape(p, g, d, 1), dtype=torch.float64, device="cuda") for d in range(2)]
    cb.face_fluxes(p, g, torch.from_numpy(Uf).cuda(), F, Fn, area_scaled=False)
    torch.cuda.synchronize()
    F = [f.cpu().numpy() for f in F]
    acc = None
    for d in range(2):
        f = F[d]
        df = (f[:, :, :, 1:] - f[:, :, :, :-1]) if d == 0 else (f[:, :, 1:, :] - f[:, :, :-1, :])
        t = df / g.dx[d]
        acc = t if acc is None else acc + t
    # the conservative components (the volume fraction carries the non-conservative term)
    np.testing.assert_array_equal(-acc[:N - 1], got[:N - 1])


@pytest.mark.parametrize("dim", [2, 3])
def test_energy_bound_min_equals_the_reference(dim):
    import torch

    p, g, U = _stressed_case(dim, "MUSCL", "air_helium_low_p")
    # some cells below the bound: lower the energy of a few cells
    V = cb.valid_view(U, p, g)
    V[2 + dim][..., 3] -= 1e-2
    got = cb.energy_bound_min(p, g, torch.from_numpy(U).cuda())
    ref = Oracle("reference", p, g).energy_bound_min(U)
    print(f"{dim}D min energy bound {got:.6e}")
    assert got == ref and got < 0


def _advance_pair(p, g, U, nsteps):
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(nsteps)
    info = lv.sync()
    got = lv.download()
    dts = lv.dts(info.steps)
    restarts = lv.bound_restarts()
    lv.close()
    ref = U.copy()
    o = Oracle("reference", p, g)
    _, dts_ref = o.advance(ref, nsteps)
    return got, info, dts, restarts, ref, dts_ref, o.bound_restarts()


# Shock-bubble runs at CFL numbers above the bounded scheme's limit (its CFL speed is about twice the
# wave speed): a step whose dt came from the last step's wave speeds violates the energy bound in a
# stage and is taken again with the general bound, which holds. Found with the oracle: 12 steps of the
# 64 x 32 bubble, one restart each.
RESTART_CASES = [
    ("MUSCL", "3.0", 0),
    ("MUSCL", "4.0", 1),
    ("MUSCL-vanLeer", "3.0", 0),
    ("WENO3", "3.5", 0),
    ("WENO5B", "3.5", 0),
]


@pytest.mark.parametrize("scheme,cfl,source_term", RESTART_CASES,
                         ids=[f"{c[0]}-cfl{c[1]}-K{c[2]}" for c in RESTART_CASES])
def test_advance_with_restarts_equals_the_reference(scheme, cfl, source_term):
    p, g, U = _bubble(scheme, {"run.cfl": cfl, "Physics.source_term": source_term}, nx=64, ny=32)
    got, info, dts, restarts, ref, dts_ref, restarts_ref = _advance_pair(p, g, U, 12)
    print(f"{scheme} cfl {cfl}: {info.steps} steps, {restarts} restarts (reference {restarts_ref}), "
          f"status {info.status}")
    assert info.status == 0 and info.steps == 12
    assert restarts == restarts_ref == 1
    np.testing.assert_array_equal(dts, dts_ref)
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))


def test_advance_stops_when_the_step_taken_again_fails():
    """MUSCL-MC at CFL 4: the step taken again with the general bound still violates it. The level keeps
    the state its failing step started from, reports COMPAS_B200_ERR_BOUND and stops; the reference's
    loop (which would go on from the violating stage state) is run to the same step."""
    p, g, U = _bubble("MUSCL-MC", {"run.cfl": "4.0"}, nx=64, ny=32)
    if not have_ref(p.physics, p.dim):
        pytest.skip("reference-header oracle not built")
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(12)
    info = lv.sync(check=False)
    got = lv.download()
    lv.close()
    assert info.status & cb.ERR_BOUND and info.steps < 12
    ref = U.copy()
    o = Oracle("reference", p, g)
    _, dts_ref = o.advance(ref, info.steps)
    assert len(dts_ref) == info.steps
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    with pytest.raises(RuntimeError):
        o.advance(U.copy(), info.steps + 1)


def test_advance_without_restarts_equals_the_reference():
    p, g, U = _bubble("WENO5", nx=64, ny=32)
    got, info, dts, restarts, ref, dts_ref, restarts_ref = _advance_pair(p, g, U, 10)
    assert info.status == 0 and restarts == restarts_ref == 0
    np.testing.assert_array_equal(dts, dts_ref)
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))


# ---- FIVEEQS_NPHASE: the reference's N-phase bounded branch (include/Operators_Compressible5Eq_NPhase/
# FVM_Conservative2FluxHyperbolic_K_Compressible5Eq_NPhase.H, Riemann_HLL_Bound_Compressible5Eq_NPhase.H),
# its MUSCL states through the consistent limiter, its WENO5B states bounding every phase
NPHASE_SCHEMES = ["GODUNOV", "MUSCL", "MUSCL-MC", "WENO3B", "WENO5", "WENO5B"]
NPHASE_CASES = {
    "triple_point": (cases.triple_point, dict(m=12)),
    "bubbles2_K": (cases.nphase_bubbles, dict(n=24, nphase=2, source_term=1, velocity=30.0)),
    "bubbles4_nasg_K": (cases.nphase_bubbles, dict(n=24, nphase=4, eos=3, source_term=1, velocity=30.0)),
    "bubbles3_3d": (cases.nphase_bubbles, dict(n=12, nphase=3, dim=3, velocity=30.0)),
    "bubbles3": (cases.nphase_bubbles, dict(n=24, nphase=3, velocity=30.0)),
}


def _nphase(name, scheme, extra=None):
    fn, kw = NPHASE_CASES[name]
    phys, dim, inputs, geom, U = fn(**kw, quadrature=False)
    inp = dict(inputs, **{"FiniteVolume.Scheme": scheme, "FiniteVolume.ID_Bound": 1}, **(extra or {}))
    p = cb.make_parm(phys, dim, inp)
    return p, cb.make_geom(**geom), U


@pytest.mark.parametrize("scheme", NPHASE_SCHEMES)
@pytest.mark.parametrize("name", list(NPHASE_CASES))
@pytest.mark.parametrize("id_lambda", [1, 0])
def test_nphase_rhs_equals_the_reference(name, scheme, id_lambda):
    p, g, U = _nphase(name, scheme)
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    p.id_lambda = id_lambda
    got, ref, cm, cm_ref, _ = _dudt_pair(p, g, U)
    np.testing.assert_array_equal(got, ref)
    assert cm == cm_ref, (cm, cm_ref)


def test_nphase_energy_bound_min_equals_the_reference():
    import torch

    p, g, U = _nphase("bubbles4_nasg_K", "MUSCL")
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    V = cb.valid_view(U, p, g)
    V[cb.parm_nstate(p) - p.nphase - 1][..., 5] -= 1e9
    got = cb.energy_bound_min(p, g, torch.from_numpy(U).cuda())
    ref = Oracle("reference", p, g).energy_bound_min(U)
    assert got == ref and got < 0


# found with the oracle: 12 steps, one restart each
NPHASE_RESTARTS = [("triple_point", "WENO5B", "3.0"), ("bubbles3", "MUSCL-MC", "2.8")]


@pytest.mark.parametrize("name,scheme,cfl", NPHASE_RESTARTS, ids=[f"{c[0]}-{c[1]}-cfl{c[2]}" for c in NPHASE_RESTARTS])
def test_nphase_advance_with_restart_equals_the_reference(name, scheme, cfl):
    p, g, U = _nphase(name, scheme, {"run.cfl": cfl})
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    got, info, dts, restarts, ref, dts_ref, restarts_ref = _advance_pair(p, g, U, 12)
    print(f"{name} {scheme} cfl {cfl}: {info.steps} steps, {restarts} restarts (reference {restarts_ref})")
    assert info.status == 0 and info.steps == 12
    assert restarts == restarts_ref == 1
    np.testing.assert_array_equal(dts, dts_ref)
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))


def test_nphase_advance_stops_when_the_step_taken_again_fails():
    p, g, U = _nphase("triple_point", "MUSCL", {"run.cfl": "2.6"})
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built")
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(12)
    info = lv.sync(check=False)
    got = lv.download()
    lv.close()
    assert info.status & cb.ERR_BOUND and info.steps < 12
    ref = U.copy()
    o = Oracle("reference", p, g)
    o.advance(ref, info.steps)
    np.testing.assert_array_equal(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    with pytest.raises(RuntimeError):
        o.advance(U.copy(), info.steps + 1)
