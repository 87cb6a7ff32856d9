"""CPU-side checks of the C ABI: the library loads, exports every declared symbol, and the inputs-key
parser follows the reference's keys, values and error behaviour (no GPU calls)."""
import os
import re

import pytest

import compas_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "compas_b200.h")).read()
    return sorted(set(re.findall(r"\b(compas_b200_[A-Za-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = cb.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(cb.EXPORTED_SYMBOLS)


def test_parm_defaults_and_eos():
    p = cb.make_parm(cb.FIVEEQS, 2, {"prob.EOS.gamma_2": 4.4, "prob.EOS.pinf_2": 6e8})
    assert p.id_limiter == 5 and p.num_grow == 3 and p.id_riemann == 2
    assert p.cfl == 0.4 and p.change_limiter == 1
    assert p.A1 == 1.0 / (1.4 - 1.0) and p.A2 == 1.0 / (4.4 - 1.0)
    assert p.B2 == 4.4 * 6e8 / (4.4 - 1.0) and p.B1 == 0.0


@pytest.mark.parametrize("key,value", [("FiniteVolume.Scheme", "WENO7"), ("Physics.RiemannSolver", "Roe"),
                                       ("prob.EOS.EOS", "7"), ("no.such.key", "1"),
                                       ("Physics.pressure_relaxation_trace", "1.5")])
def test_invalid_inputs_are_errors_not_aborts(key, value):
    with pytest.raises(cb.CompasError) as e:
        cb.make_parm(cb.FIVEEQS, 2, {key: value})
    assert e.value.code == cb.EARG


def test_scheme_keys():
    """FiniteVolume.Scheme to the reference's ID_WENO / ID_Limiter / Num_Grow
    (include/Operators_FV/FiniteVolume_Parameter.H:51-147)."""
    p = cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.Scheme": "WENO5B"})
    assert (p.id_weno, p.id_limiter, p.num_grow) == (1, 6, 3)
    for v, lim, ng in [("GODUNOV", 0, 1), ("MUSCL", 1, 2), ("MUSCL-Minmod", 1, 2), ("MUSCL-vanLeer", 2, 2),
                       ("MUSCL-Superbee", 3, 2), ("MUSCL-MC", 4, 2)]:
        p = cb.make_parm(cb.SIXEQS, 3, {"FiniteVolume.Scheme": v})
        assert (p.id_weno, p.id_limiter, p.num_grow) == (0, lim, ng), v
    p = cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.Scheme": "WENO3"})
    assert (p.id_weno, p.id_limiter, p.num_grow) == (1, 3, 2)
    p = cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.Scheme": "WENO3B"})
    assert (p.id_weno, p.id_limiter, p.num_grow) == (1, 4, 2)


def test_state_bytes_layout():
    p = cb.make_parm(cb.SIXEQS, 3, {})
    g = cb.make_geom((10, 12, 14), (1, 1, 1), 3)
    assert cb.padded_shape(p, g) == (8, 20, 18, 16)
    assert cb.lib().compas_b200_state_bytes(p, g) == 8 * 20 * 18 * 16 * 8


def test_autotune_key():
    assert cb.make_parm(cb.FIVEEQS, 2).autotune == 1
    assert cb.make_parm(cb.FIVEEQS, 2, {"compas_b200.autotune": 0}).autotune == 0
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS, 2, {"compas_b200.autotune": 2})


def test_tma_key():
    assert cb.make_parm(cb.SIXEQS, 3).tma == 1
    assert cb.make_parm(cb.SIXEQS, 3, {"compas_b200.tma": 0}).tma == 0
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.SIXEQS, 3, {"compas_b200.tma": 3})


def test_phase_field_formulation_key():
    """PhaseField.ID_FluxPhase2Flux: the mixture formulation by default for FIVEEQS
    (include/Physics_PhaseField/PhaseField_Parameter.H:53), the phasic one for SIXEQS
    (exec/_Tests/Advection/prob/Parm.H:48-50); both models take both."""
    assert cb.make_parm(cb.FIVEEQS, 2).pf_phase2flux == 1
    assert cb.make_parm(cb.SIXEQS, 3).pf_phase2flux == 0
    assert cb.make_parm(cb.SIXEQS, 2, {"PhaseField.ID_FluxPhase2Flux": 1}).pf_phase2flux == 1
    assert cb.make_parm(cb.FIVEEQS, 3, {"PhaseField.ID_FluxPhase2Flux": 1}).pf_phase2flux == 1
    assert cb.make_parm(cb.FIVEEQS, 2, {"PhaseField.ID_FluxPhase2Flux": 0}).pf_phase2flux == 0
    with pytest.raises(cb.CompasError) as e:
        cb.make_parm(cb.SIXEQS, 2, {"PhaseField.ID_FluxPhase2Flux": 2})
    assert e.value.code == cb.EARG
    assert cb.make_parm(cb.SIXEQS, 2).pf_flux == 0
    assert cb.make_parm(cb.SIXEQS, 2, {"PhaseField.ID_Flux": 1}).pf_flux == 1
    assert cb.make_parm(cb.FIVEEQS, 2, {"PhaseField.ID_Flux": 1}).pf_flux == 1
    with pytest.raises(cb.CompasError) as e:
        cb.make_parm(cb.FIVEEQS, 2, {"PhaseField.ID_Flux": 2})
    assert e.value.code == cb.EARG


def test_nc_terms_and_face_shapes():
    """NC_TERMS of include/Macros.H per model, and the face-array shapes of the flux-register entry
    point (a face MultiFab without ghosts: one more face than cells along its direction)."""
    assert cb.nc_terms(cb.make_parm(cb.FIVEEQS, 2, {})) == 1
    assert cb.nc_terms(cb.make_parm(cb.SIXEQS, 3, {})) == 3
    assert cb.nc_terms(cb.make_parm(cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4, 1.5, 1.6]})) == 1
    p = cb.make_parm(cb.SIXEQS, 3, {})
    g = cb.make_geom((5, 6, 7), (0.1, 0.1, 0.1))
    assert cb.face_shape(p, g, 0, 8) == (8, 7, 6, 6)
    assert cb.face_shape(p, g, 1, 3) == (3, 7, 7, 5)
    assert cb.face_shape(p, g, 2, 8) == (8, 8, 6, 5)


def test_amr_interpolater_key():
    """amr.Interpolater: lincc_interp (default) and pc_interp; quartic_interp is refused, an unknown value
    is an error naming the valid ones (source/COMPAS.cpp:1217-1221)."""
    assert cb.make_parm(cb.FIVEEQS, 2, {}).amr_interp == 0
    assert cb.make_parm(cb.FIVEEQS, 2, {"amr.Interpolater": "pc_interp"}).amr_interp == 1
    with pytest.raises(cb.CompasError) as e:
        cb.make_parm(cb.FIVEEQS, 2, {"amr.Interpolater": "cubic"})
    assert "pc_interp, lincc_interp, quartic_interp" in str(e.value)
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS, 2, {"amr.Interpolater": "quartic_interp"})


def test_bound_preserving_key():
    """FiniteVolume.ID_Bound (FiniteVolume_Parameter.H:45, :56): 0 / 1, ID_Lambda starting at 1; the bounded
    branch is the five-equation models', in FP64, without the Phase-Field step (the checks run before any
    device call, so they hold without a GPU)."""
    p = cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.ID_Bound": 1, "FiniteVolume.Scheme": "MUSCL-MC"})
    assert p.id_bound == 1 and p.id_lambda == 1
    assert cb.make_parm(cb.FIVEEQS, 3, {}).id_bound == 0
    with pytest.raises(cb.CompasError):
        cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.ID_Bound": 2})
    g = cb.make_geom((16, 16, 1), (0.1, 0.1, 1.0))
    g3 = cb.make_geom((8, 8, 8), (0.1, 0.1, 0.1))
    for phys, dim, extra, geom in [(cb.SIXEQS, 3, {}, g3), (cb.FIVEEQS, 2, {"compas_b200.precision": "mixed"}, g),
                                   (cb.FIVEEQS_NPHASE, 2, {"prob.EOS.gamma": [1.4, 1.5, 1.6],
                                                           "PhaseField.phase_field": 1}, g)]:
        q = cb.make_parm(phys, dim, dict({"FiniteVolume.ID_Bound": 1}, **extra))
        with pytest.raises(cb.CompasError) as e:
            cb.Level(q, geom)
        assert e.value.code == cb.EUNSUPPORTED
    with pytest.raises(cb.CompasError) as e:
        cb.energy_bound_min(cb.make_parm(cb.SIXEQS, 3, {}), g3, None, out=0)
    assert e.value.code in (cb.EUNSUPPORTED, cb.EARG)


def test_sixeqs_ie_nphase_keys():
    """SIXEQS_IE_NPHASE (include/Macros.H:59): NSTATE = 3 NPHASE + dim + 1, the per-phase EOS lists of
    the N-phase Parm (source/Parm.cpp:364-446), pressure relaxation keys; the engine runs it in FP64
    on the single-level API with NPHASE 2, 3 in 2D and 3 in 3D (the checks run before any device call)."""
    inputs = {"prob.EOS.gamma": [4.4, 1.4, 1.667], "prob.EOS.pinf": [6e8, 0.0, 0.0],
              "Physics.pressure_relaxation": 1, "Physics.pressure_relaxation_trace": 1e-3,
              "FiniteVolume.Scheme": "MUSCL"}
    p = cb.make_parm(cb.SIXEQS_IE_NPHASE, 2, inputs)
    assert p.nphase == 3 and cb.parm_nstate(p) == 12 and cb.nstate(cb.SIXEQS_IE_NPHASE, 3, 3) == 13
    assert p.relaxation == 1 and p.relax_trace == 1e-3
    assert abs(p.Ak[0] - 1.0 / 3.4) < 1e-15 and abs(p.Bk[0] - 4.4 * 6e8 / 3.4) < 1e-6 and p.Bk[1] == 0.0
    assert cb.nc_terms(p) == 1
    g = cb.make_geom((16, 16, 1), (0.1, 0.1, 1.0))
    g3 = cb.make_geom((8, 8, 8), (0.1, 0.1, 0.1))
    bad = [(2, dict(inputs, **{"FiniteVolume.THINC": 1, "FiniteVolume.Scheme": "WENO5"}), g),
           (2, dict(inputs, **{"FiniteVolume.ID_Bound": 1}), g),
           (2, dict(inputs, **{"prob.EOS.gamma": [1.4] * 4, "prob.EOS.pinf": [0.0] * 4}), g),
           (3, dict(inputs, **{"prob.EOS.gamma": [1.4] * 2, "prob.EOS.pinf": [0.0] * 2}), g3)]
    for dim, inp, geom in bad:
        q = cb.make_parm(cb.SIXEQS_IE_NPHASE, dim, inp)
        with pytest.raises(cb.CompasError) as e:
            cb.Level(q, geom)
        assert e.value.code == cb.EUNSUPPORTED
    with pytest.raises(cb.CompasError) as e:
        cb.Batch(cb.SIXEQS_IE_NPHASE, 2, 5, 1, 4, nphase=4)  # NPHASE 4 is not compiled for this model
    assert e.value.code == cb.EUNSUPPORTED
