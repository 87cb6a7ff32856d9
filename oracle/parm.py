"""Test infrastructure: the oracle's own reading of the inputs keys into an oracle Case, so that a CPU
run of the reference arithmetic (the reference arm of bench.py) needs nothing from the CUDA library.

Restates, for the two-phase models (FIVEEQS, SIXEQS):
  * source/Parm.cpp:101-188 - the EOS coefficients A, B, C, D of ideal gas (EOS 0), stiffened gas
    (EOS 1) and NASG (EOS 3: covolume b in C, heat of formation q in D) from prob.EOS.*;
  * include/Operators_FV/FiniteVolume_Parameter.H:51-147 - FiniteVolume.Scheme to (ID_Limiter,
    ID_WENO);
  * source/Class_Compressible_PhaseField.cpp:92-111 - Physics.RiemannSolver to its id (LLF 0, HLL 1,
    HLLC 2);
  * the defaults of run.cfl (0.4), run.timestep_change_limiter (1), Physics.source_term (0), the THINC keys
    (include/Operators_FV/FiniteVolume_Parameter.H).
Only tests and the CPU legs of bench.py use this module; the product never imports it.
"""
from __future__ import annotations

from .oracle import FIVEEQS, SIXEQS, Case

SCHEMES = {"WENO5": (5, 1), "WENO5B": (6, 1), "GODUNOV": (0, 0), "MUSCL": (1, 0), "MUSCL-Minmod": (1, 0),
           "MUSCL-vanLeer": (2, 0), "MUSCL-Superbee": (3, 0), "MUSCL-MC": (4, 0), "WENO3": (3, 1),
           "WENO3B": (4, 1)}
RIEMANN = {"LLF": 0, "HLL": 1, "HLLC": 2}


def eos_coefficients(eos: int, gamma: float, pinf: float = 0.0, b: float = 0.0, q: float = 0.0):
    """(A, B, C, D) of one phase, source/Parm.cpp:120-150."""
    if not gamma > 1.0:
        raise ValueError("prob.EOS.EOS requires gamma > 1")
    A = 1.0 / (gamma - 1.0)
    if eos == 0:
        return A, 0.0, 0.0, 0.0
    if eos == 1:
        return A, gamma * pinf / (gamma - 1.0), 0.0, 0.0
    if eos == 3:
        if b < 0.0:
            raise ValueError("prob.EOS.b must be >= 0")
        return A, gamma * pinf / (gamma - 1.0), b, q
    raise ValueError(f"prob.EOS.EOS = {eos} is not supported by the oracle (0, 1, 3)")


def reference_case(physics: int, dim: int, inputs: dict, geom: dict) -> Case:
    """Oracle Case of a two-phase model from inputs keys and a geometry dict (n, dx, ng, lo_bc, hi_bc)."""
    if physics not in (FIVEEQS, SIXEQS):
        raise ValueError("the oracle's own Parm covers FIVEEQS and SIXEQS")
    g = lambda k, d: inputs.get(k, d)  # noqa: E731
    c = Case()
    c.physics, c.dim = physics, dim
    for d in range(3):
        c.n[d] = int(geom["n"][d]) if d < dim else 1
        c.dx[d] = float(geom["dx"][d])
        c.lo_bc[d] = int(geom["lo_bc"][d])
        c.hi_bc[d] = int(geom["hi_bc"][d])
    c.ng = int(geom["ng"])
    eos = int(g("prob.EOS.EOS", 1))
    c.A1, c.B1, c.C1, c.D1 = eos_coefficients(eos, float(g("prob.EOS.gamma_1", 1.4)), float(g("prob.EOS.pinf_1", 0.0)),
                                              float(g("prob.EOS.b_1", 0.0)), float(g("prob.EOS.q_1", 0.0)))
    c.A2, c.B2, c.C2, c.D2 = eos_coefficients(eos, float(g("prob.EOS.gamma_2", 1.4)), float(g("prob.EOS.pinf_2", 0.0)),
                                              float(g("prob.EOS.b_2", 0.0)), float(g("prob.EOS.q_2", 0.0)))
    scheme = str(g("FiniteVolume.Scheme", "WENO5"))
    if scheme not in SCHEMES:
        raise ValueError(f"FiniteVolume.Scheme = '{scheme}' is not recognized")
    c.id_limiter, c.id_weno = SCHEMES[scheme]
    c.id_riemann = RIEMANN[str(g("Physics.RiemannSolver", "HLLC"))]
    c.source_term = int(g("Physics.source_term", 0))
    c.relaxation = 1 if int(g("Physics.pressure_relaxation", 0)) else 0
    c.relax_trace = float(g("Physics.pressure_relaxation_trace", 0.0))
    c.thinc = int(g("FiniteVolume.THINC", 0))
    c.thinc_use_normal = int(g("FiniteVolume.THINC.UseNormal", 1))
    c.thinc_eps = float(g("FiniteVolume.THINC.EPS", 1e-4))
    c.thinc_beta = float(g("FiniteVolume.THINC.Beta", 2.3))
    c.thinc_normal_threshold = float(g("FiniteVolume.THINC.NormalThreshold", 0.25))
    c.cfl = float(g("run.cfl", 0.4))
    c.change_limiter = 1 if int(g("run.timestep_change_limiter", 1)) else 0
    c.nphase = 2
    c.amr_interp = {"lincc_interp": 0, "pc_interp": 1}[str(g("amr.Interpolater", "lincc_interp"))]
    # FiniteVolume.ID_Bound (FiniteVolume_Parameter.H:45, :56); ID_Lambda starts at its default 1 (:47)
    c.id_bound = int(g("FiniteVolume.ID_Bound", 0))
    c.id_lambda = 1
    return c
