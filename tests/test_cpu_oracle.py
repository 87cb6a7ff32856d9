"""CPU checks of the oracle: the plain-C restatement is pinned to the reference's own arithmetic
(the golden fixtures made from the reference-header build, and that build itself where present),
and both satisfy the invariants the reference's tests rely on (conservation, equilibrium
preservation, NASG with b = 0 equal to the stiffened gas)."""
import ast
import glob
import os

import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from oracle.oracle import Oracle, have_ref

GOLDEN_ALL = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
# the plain-C restatement covers FIVEEQS, SIXEQS and FIVEEQS_NPHASE; SIXEQS_IE_NPHASE is pinned through
# the reference-header build only
GOLDEN = [p for p in GOLDEN_ALL if "_6eqn" not in os.path.basename(p)]
GOLDEN_SIXN = [p for p in GOLDEN_ALL if "_6eqn" in os.path.basename(p)]


def _parm_geom(physics, dim, inputs, geom):
    return cb.make_parm(physics, dim, inputs), cb.make_geom(**geom)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_port_matches_reference_golden(path):
    z = np.load(path)
    phys, dim, steps = (int(x) for x in z["physics"])
    p, g = _parm_geom(phys, dim, ast.literal_eval(str(z["inputs"])), ast.literal_eval(str(z["geom"])))
    U = z["U0"].copy()
    t, dts = Oracle("port", p, g).advance(U, steps)
    np.testing.assert_array_equal(dts, z["dts"])
    assert t == float(z["t"][0])
    np.testing.assert_array_equal(cb.valid_view(U, p, g), z["valid"])


@pytest.mark.parametrize("path", GOLDEN_SIXN, ids=[os.path.basename(p) for p in GOLDEN_SIXN])
def test_reference_build_reproduces_sixn_golden(path):
    """The SIXEQS_IE_NPHASE fixtures against the reference-header build that made them (a rebuilt
    oracle/_ref must give the same bits)."""
    z = np.load(path)
    phys, dim, steps = (int(x) for x in z["physics"])
    p, g = _parm_geom(phys, dim, ast.literal_eval(str(z["inputs"])), ast.literal_eval(str(z["geom"])))
    if not have_ref(p.physics, p.dim, p.nphase):
        pytest.skip("reference-header oracle not built here")
    U = z["U0"].copy()
    t, dts = Oracle("reference", p, g).advance(U, steps)
    np.testing.assert_array_equal(dts, z["dts"])
    np.testing.assert_array_equal(cb.valid_view(U, p, g), z["valid"])


@pytest.mark.skipif(not have_ref(cb.FIVEEQS, 2), reason="reference-header oracle not built here")
@pytest.mark.parametrize("case,kw,steps,extra", [
    (cases.advected_disc, dict(n=40), 8, {}),
    (cases.shock_bubble, dict(nx=33, ny=21, scheme="WENO5"), 8, {}),
    (cases.shock_droplet, dict(n=14), 2, {}),
    (cases.advected_disc, dict(n=40), 8, {"FiniteVolume.THINC": "1"}),
    (cases.advected_disc, dict(n=36), 8, {"FiniteVolume.THINC": "1", "FiniteVolume.THINC.UseNormal": "0"}),
    (cases.shock_bubble, dict(nx=33, ny=21, scheme="WENO5B"), 8, {"FiniteVolume.THINC": "1"}),
    (cases.shock_droplet, dict(n=14), 2, {"FiniteVolume.THINC": "1"}),
])
def test_port_matches_reference_build(case, kw, steps, extra):
    phys, dim, inputs, geom, U = case(**kw)
    inputs = dict(inputs, **extra)
    p, g = _parm_geom(phys, dim, inputs, geom)
    a, b = U.copy(), U.copy()
    ta, da = Oracle("reference", p, g).advance(a, steps)
    tb, db = Oracle("port", p, g).advance(b, steps)
    np.testing.assert_array_equal(da, db)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("case,kw,steps", [
    (cases.triple_point, dict(m=8), 12),
    (cases.nphase_bubbles, dict(n=20, nphase=2), 6),
    (cases.nphase_bubbles, dict(n=20, nphase=3, source_term=1), 6),
    (cases.nphase_bubbles, dict(n=20, nphase=4, eos=3, source_term=1), 6),
    (cases.nphase_bubbles, dict(n=10, nphase=3, dim=3), 2),
], ids=["triple8", "bubbles2", "bubbles3_K", "bubbles4_nasg_K", "bubbles3_3d"])
def test_port_matches_reference_build_nphase(case, kw, steps):
    """The N-phase restatement (WENO5 with the consistent limiter, HLLC, Kapila terms) equals the
    reference's own N-phase headers to the bit."""
    phys, dim, inputs, geom, U = case(**kw)
    p, g = _parm_geom(phys, dim, inputs, geom)
    if not have_ref(phys, dim, p.nphase):
        pytest.skip("reference-header oracle not built here")
    a, b = U.copy(), U.copy()
    ta, da = Oracle("reference", p, g).advance(a, steps)
    tb, db = Oracle("port", p, g).advance(b, steps)
    np.testing.assert_array_equal(da, db)
    np.testing.assert_array_equal(a, b)


def test_nphase_parm_lists_follow_the_reference_rules():
    """prob.EOS.gamma and the other per-phase lists need exactly NPHASE values (source/Parm.cpp:82-92);
    A_k = 1/(gamma_k - 1), B_k = gamma_k pinf_k/(gamma_k - 1)."""
    p = cb.make_parm(cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4, 1.5, 4.4], "prob.EOS.pinf": [0, 0, 6e8]})
    assert p.nphase == 3 and cb.parm_nstate(p) == 9
    assert list(p.Ak[:3]) == [1.0 / (1.4 - 1.0), 1.0 / (1.5 - 1.0), 1.0 / (4.4 - 1.0)]
    assert p.Bk[2] == 4.4 * 6e8 / (4.4 - 1.0)
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4, 1.5]}, nphase=3)
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4, 0.9, 1.5]})
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4] * 5}, nphase=5)


def test_conservation_periodic_round_off():
    phys, dim, inputs, geom, U = cases.advected_disc(n=32)
    p, g = _parm_geom(phys, dim, inputs, geom)
    V0 = cb.valid_view(U, p, g).copy()
    Oracle("port", p, g).advance(U, 10)
    V = cb.valid_view(U, p, g)
    for c in range(5):  # masses, momenta, total energy
        s0 = V0[c].sum()
        assert abs(V[c].sum() - s0) <= 1e-13 * np.abs(V0[c]).sum()


def test_uniform_pressure_velocity_equilibrium_is_kept():
    """Uniform p and u across a material interface stay uniform (the Advection test's equilibrium
    errors): the five-equation WENO5 + HLLC scheme in primitive variables keeps them to round-off."""
    phys, dim, inputs, geom, U = cases.advected_disc(n=32)
    p, g = _parm_geom(phys, dim, inputs, geom)
    o = Oracle("port", p, g)
    o.advance(U, 10)
    V = cb.valid_view(U, p, g)
    rho = V[0] + V[1]
    u, v = V[2] / rho, V[3] / rho
    assert np.max(np.abs(u - 1.0)) < 1e-9 and np.max(np.abs(v - 1.0)) < 1e-9
    a1 = V[5]
    pres = (V[4] - 0.5 * rho * (u * u + v * v) - (1 - a1) * p.B2) / (a1 * p.A1 + (1 - a1) * p.A2)
    assert np.max(np.abs(pres / 1e5 - 1.0)) < 1e-7


def test_nasg_with_zero_covolume_equals_stiffened_gas():
    """prob.EOS.EOS = 3 with b = q = 0 is bit-identical to EOS = 1 (the eos-nasg-b0 variants)."""
    phys, dim, inputs, geom, U = cases.shock_droplet(n=10)
    p1, g = _parm_geom(phys, dim, inputs, geom)
    p3, _ = _parm_geom(phys, dim, dict(inputs, **{"prob.EOS.EOS": 3}), geom)
    a, b = U.copy(), U.copy()
    Oracle("port", p1, g).advance(a, 2)
    Oracle("port", p3, g).advance(b, 2)
    np.testing.assert_array_equal(a, b)


def test_mirror_symmetry_of_the_droplet():
    """The droplet case is symmetric in y about the centre plane; the scheme keeps it up to rounding,
    which the epsilon-free WENO5 weight ratios amplify to ~1e-10 relative."""
    phys, dim, inputs, geom, U = cases.shock_droplet(n=12)
    p, g = _parm_geom(phys, dim, inputs, geom)
    Oracle("port", p, g).advance(U, 2)
    V = cb.valid_view(U, p, g)
    for c in (0, 1, 2, 5, 6, 7):
        np.testing.assert_allclose(V[c], V[c][:, ::-1, :], rtol=1e-8, atol=1e-8 * np.abs(V[c]).max())


def _amr_run(max_grid_size, steps=3):
    from compas_b200 import amr

    kw = dict(nx=64, ny=32, scheme="WENO5B")
    phys, dim, inputs, geom, _ = cases.shock_bubble(**kw)
    p, g = _parm_geom(phys, dim, inputs, geom)
    regions = [((40, 16, 0), (95, 47, 0)), ((96, 48, 0), (175, 79, 0))]
    boxes = amr.hierarchy((64, 32), dim, regions, max_grid_size)
    states = amr.box_states(cases.shock_bubble, kw, (64, 32), dim, boxes)
    _, dts = Oracle("reference", p, g).amr_advance(boxes, states, steps)
    # each level as one array
    out = {}
    for (lev, lo, hi), S in zip(boxes, states):
        scale = 1 << lev
        a = out.setdefault(lev, np.full((S.shape[0], 32 * scale, 64 * scale), np.nan))
        a[:, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = S[:, 0, 3:3 + hi[1] - lo[1] + 1, 3:3 + hi[0] - lo[0] + 1]
    return dts, out


@pytest.mark.skipif(not have_ref(cb.FIVEEQS, 2), reason="reference-header oracle not built here")
def test_amr_oracle_independent_of_box_decomposition():
    dts_a, a = _amr_run(32)
    dts_b, b = _amr_run(8)
    np.testing.assert_array_equal(dts_a, dts_b)
    for lev in a:
        np.testing.assert_array_equal(a[lev], b[lev])


@pytest.mark.skipif(not have_ref(cb.FIVEEQS, 2), reason="reference-header oracle not built here")
def test_amr_oracle_conserves_composite_totals_periodic():
    from compas_b200 import amr

    kw = dict(n=32)
    phys, dim, inputs, geom, _ = cases.advected_disc(**kw)
    p, g = _parm_geom(phys, dim, inputs, geom)
    boxes = amr.hierarchy((32, 32), 2, [((16, 16, 0), (47, 47, 0)), ((40, 40, 0), (87, 87, 0))], 16)
    states = amr.box_states(cases.advected_disc, kw, (32, 32), 2, boxes)
    cov = amr.covered_mask_fn(boxes, 2)
    s0 = [amr.composite_sum(states, boxes, 2, 3, c, cov) for c in range(5)]
    Oracle("reference", p, g).amr_advance(boxes, states, 6)
    s1 = [amr.composite_sum(states, boxes, 2, 3, c, cov) for c in range(5)]
    for a, b in zip(s0, s1):
        assert abs(a - b) <= 1e-13 * abs(a)


@pytest.mark.parametrize("form,flux", [("0", "0"), ("1", "0"), ("0", "1"), ("1", "1")])
def test_sixeq_phase_field_oracle_keeps_equilibrium_and_conserves(form, flux):
    """The six-equation Phase-Field step of the reference-header build (phasic 0 / mixture 1
    formulation, upwind/downwind 0 / HLL 1 phase fluxes, CAC-Adv with the elliptic solve, relaxation
    after every stage) keeps a uniform
    velocity and pressure across the interface and conserves the masses, momenta and total energy."""
    phys, dim, inputs, geom, U = cases.advected_interface(n=32, dim=2, physics=cb.SIXEQS)
    p, g = _parm_geom(phys, dim, dict(inputs, **{"PhaseField.phase_field": "1", "LinearSystem.tol_rel": "1e-13",
                                                 "PhaseField.ID_FluxPhase2Flux": form, "PhaseField.ID_Flux": flux}),
                      geom)
    if not have_ref(p.physics, p.dim):
        pytest.skip("reference-header oracle not built")
    from oracle.oracle import pf_from

    V0 = cb.valid_view(U, p, g).copy()
    Oracle("reference", p, g).advance_pf(U, pf_from(p), 3)
    V = cb.valid_view(U, p, g)
    rho = V[0] + V[1]
    u, v = V[2] / rho, V[3] / rho
    a1 = V[6]
    k = 0.5 * (u * u + v * v)
    pres = (V[4] - V[0] * k - a1 * p.B1) / p.A1 + (V[5] - V[1] * k - (1 - a1) * p.B2) / p.A2
    assert np.max(np.abs(u - 1.0)) < 1e-8 and np.max(np.abs(v - 1.0)) < 1e-8
    assert np.max(np.abs(pres / 1e5 - 1.0)) < 1e-7
    for c in range(4):
        assert abs(V[c].sum() - V0[c].sum()) <= 1e-13 * np.abs(V0[c]).sum(), c
    E0 = V0[4].sum() + V0[5].sum()
    assert abs(V[4].sum() + V[5].sum() - E0) <= 1e-12 * abs(E0)


@pytest.mark.skipif(not have_ref(cb.SIXEQS, 2), reason="reference-header oracle not built here")
def test_sixeq_amr_oracle_conserves_composite_totals_periodic():
    """Six-equation multi-level advance of the oracle (flux registers with the three non-conservative
    face terms, the phase-energy reflux source terms, relaxation of the refluxed cells): the composite
    masses, momenta and total energy (the sum of the phase energies) are conserved on a periodic square."""
    from compas_b200 import amr

    kw = dict(n=16, dim=2, physics=cb.SIXEQS)
    phys, dim, inputs, geom, _ = cases.advected_interface(**kw)
    p, g = _parm_geom(phys, dim, inputs, geom)
    boxes = amr.hierarchy((16, 16), 2, [((8, 8, 0), (23, 23, 0))], 8)
    states = amr.box_states(cases.advected_interface, kw, (16, 16), 2, boxes)
    cov = amr.covered_mask_fn(boxes, 2)

    def totals(st):
        s = [amr.composite_sum(st, boxes, 2, 3, c, cov) for c in range(6)]
        return s[:4] + [s[4] + s[5]]

    s0 = totals(states)
    Oracle("reference", p, g).amr_advance(boxes, states, 4)
    s1 = totals(states)
    for a, b in zip(s0, s1):
        assert abs(a - b) <= 1e-13 * abs(a)


@pytest.mark.parametrize("scheme", ["GODUNOV", "MUSCL", "MUSCL-vanLeer", "MUSCL-Superbee", "MUSCL-MC", "WENO3"])
def test_muscl_reference_oracle_conserves_and_keeps_equilibrium(scheme):
    """The reference-header oracle with the GODUNOV / MUSCL reconstructions: conservation on the periodic
    square and the uniform pressure and velocity across the interface kept (the five-equation
    primitive-variable reconstruction)."""
    phys, dim, inputs, geom, U = cases.advected_disc(n=32)
    p, g = _parm_geom(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": scheme}), geom)
    if not have_ref(p.physics, p.dim):
        pytest.skip("reference-header oracle not built")
    V0 = cb.valid_view(U, p, g).copy()
    Oracle("reference", p, g).advance(U, 10)
    V = cb.valid_view(U, p, g)
    for c in range(5):
        assert abs(V[c].sum() - V0[c].sum()) <= 1e-13 * np.abs(V0[c]).sum(), c
    rho = V[0] + V[1]
    u, v = V[2] / rho, V[3] / rho
    assert np.max(np.abs(u - 1.0)) < 1e-9 and np.max(np.abs(v - 1.0)) < 1e-9


def test_port_rejects_the_muscl_family():
    """The plain-C restatement covers WENO5 / WENO5B; it refuses the other schemes."""
    phys, dim, inputs, geom, U = cases.advected_disc(n=16)
    p, g = _parm_geom(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": "MUSCL-MC"}), geom)
    with pytest.raises(RuntimeError):
        Oracle("port", p, g).advance(U, 1)


@pytest.mark.skipif(not have_ref(cb.FIVEEQS_NPHASE, 2, 3), reason="reference-header oracle not built here")
def test_nphase_amr_oracle_conserves_masses_and_energy():
    """N-phase (NPHASE 3) multi-level advance of the oracle on the triple point with the MUSCL-MC of its
    example (flux registers, the per-phase alpha_k reflux source terms): behind reflecting walls the
    composite masses and total energy are conserved to round-off."""
    from compas_b200 import amr

    kw = dict(m=8)
    phys, dim, inputs, geom, _ = cases.triple_point(**kw)
    p, g = _parm_geom(phys, dim, dict(inputs, **{"FiniteVolume.Scheme": "MUSCL-MC"}), geom)
    boxes = amr.hierarchy((56, 24), 2, [((8, 8, 0), (47, 39, 0)), ((24, 24, 0), (71, 55, 0))], 16)
    states = amr.box_states(cases.triple_point, kw, (56, 24), 2, boxes)
    cov = amr.covered_mask_fn(boxes, 2)
    comps = (0, 1, 2, 5)  # the three partial densities, the total energy
    s0 = [amr.composite_sum(states, boxes, 2, 3, c, cov) for c in comps]
    Oracle("reference", p, g).amr_advance(boxes, states, 4)
    s1 = [amr.composite_sum(states, boxes, 2, 3, c, cov) for c in comps]
    for a, b in zip(s0, s1):
        assert abs(a - b) <= 1e-13 * abs(a)


def test_oracle_parm_matches_the_library_parm():
    """The oracle's own reading of the inputs keys (oracle/parm.py, used by the CPU legs of bench.py
    so that they load no CUDA library) gives the same oracle Case as the library's Parm."""
    from oracle.oracle import case_from
    from oracle.parm import reference_case

    variants = [cases.shock_droplet(n=8), cases.shock_bubble(nx=16, ny=8), cases.advected_disc(n=8)]
    phys, dim, inputs, geom, _ = cases.shock_bubble(nx=16, ny=8, scheme="MUSCL-MC")
    variants.append((phys, dim, dict(inputs, **{"Physics.RiemannSolver": "HLL", "run.timestep_change_limiter": 0,
                                                 "FiniteVolume.THINC": 1, "Physics.source_term": 1}), geom, None))
    nasg = {"prob.EOS.EOS": 3, "prob.EOS.gamma_1": 1.19, "prob.EOS.gamma_2": 1.19, "prob.EOS.pinf_2": 6.2178e8,
            "prob.EOS.b_2": 6.7212e-4, "prob.EOS.q_2": -1.177788e6}
    variants.append((cb.FIVEEQS, 2, nasg, geom, None))
    for phys, dim, inputs, geom, _ in variants:
        a = reference_case(phys, dim, inputs, geom)
        b = case_from(cb.make_parm(phys, dim, inputs), cb.make_geom(**geom))
        for name, _t in a._fields_:
            va, vb = getattr(a, name), getattr(b, name)
            if hasattr(va, "__len__"):
                va, vb = list(va), list(vb)
            if name in ("Ak", "Bk", "Ck", "Dk"):
                continue  # N-phase only
            assert va == vb, (name, va, vb, inputs)
