// Test infrastructure (oracle): the per-case parameter struct that the reference's physics headers
// take as `Parm const&`. Field names and meanings mirror exec/_Tests/Advection/prob/Parm.H:33-117
// (the two-phase models), exec/TriplePoint-5Eq-N/prob/Parm.H (FIVEEQS_NPHASE) and
// exec/ShockBubble-WaterAir-6Eq-Nphase/prob/Parm.H (SIXEQS_IE_NPHASE); the linear-solver block is left out because no hyperbolic-path function
// reads it. The oracle driver fills the fields directly (the EOS coefficients as source/Parm.cpp:
// 101-188 computes them), so no ParmParse input is read.
#ifndef PARM_H_
#define PARM_H_

#include <AMReX_REAL.H>
#include <AMReX_Array.H>
#include <Macros.H>

#if (PHYSICS == FIVEEQS)
#include <Physics_Parameter_Compressible5Eq.H>
#elif (PHYSICS == SIXEQS)
#include <Physics_Parameter_Compressible6Eq.H>
#elif (PHYSICS == FIVEEQS_NPHASE)
#include <Physics_Parameter_Compressible5Eq_NPhase.H>
#elif (PHYSICS == SIXEQS_IE_NPHASE)
#include <Physics_Parameter_Compressible6Eq_IE_NPhase.H>
#else
#error "the oracle build covers FIVEEQS, SIXEQS, FIVEEQS_NPHASE and SIXEQS_IE_NPHASE"
#endif
#include <FiniteVolume_Parameter.H>
#include <PhaseField_Parameter.H>

#if (PHYSICS == FIVEEQS_NPHASE || PHYSICS == SIXEQS_IE_NPHASE)
// The N-phase models' Parm (exec/TriplePoint-5Eq-N/prob/Parm.H,
// exec/ShockBubble-WaterAir-6Eq-Nphase/prob/Parm.H): per-phase EOS arrays.
struct Parm
{
    Physics_Parameter Physics_Parm;
    FiniteVolume_Parameter FiniteVolume_Parm;
    PhaseField_Parameter PhaseField_Parm;

    int EOS = 1;
    amrex::Array<amrex::Real, NPHASE> A, B, C, D;
    amrex::Array<amrex::Real, NPHASE> gamma, pinf, gGamma, pref, eref, cv, mu, muB, kappa;

    amrex::Real K = 0.0;
    amrex::Array<amrex::Real, NSTATE> UpperBound;
    amrex::Array<amrex::Real, NSTATE> LowerBound;
    amrex::Array<int, NSTATE> ID_BoundType;
    amrex::Array<amrex::Real, NPHASE> p_min;
    int interface_thickness = 0;
};
#else
struct Parm
{
    Physics_Parameter Physics_Parm;
    FiniteVolume_Parameter FiniteVolume_Parm;
#if (PHYSICS == SIXEQS)
    // the six-equation model's Parm.H selects the phasic formulation of the Phase-Field fluxes
    PhaseField_Parameter PhaseField_Parm{.ID_FluxPhase2Flux = 0};
#else
    PhaseField_Parameter PhaseField_Parm;
#endif

    int EOS = 1;

    amrex::Real gamma_1 = 1.4;
    amrex::Real gamma_2 = 1.4;
    amrex::Real pinf_1 = 0.0, pinf_2 = 0.0;
    amrex::Real gGamma_1 = 0.0, gGamma_2 = 0.0, pref_1 = 0.0, pref_2 = 0.0, eref_1 = 0.0, eref_2 = 0.0;
    amrex::Real cv_1 = 1.0, cv_2 = 1.0;
    amrex::Real mu_1 = 0.0, mu_2 = 0.0, muB_1 = 0.0, muB_2 = 0.0, kappa_1 = 0.0, kappa_2 = 0.0;

    amrex::Real A1 = 0, A2 = 0, B1 = 0, B2 = 0, C1 = 0, C2 = 0, D1 = 0, D2 = 0;

    amrex::Real K = 0.0;
    amrex::Array<amrex::Real, NSTATE> UpperBound;
    amrex::Array<amrex::Real, NSTATE> LowerBound;
    amrex::Array<int, NSTATE> ID_BoundType;
    amrex::Array<amrex::Real, 2> p_min;
    int interface_thickness = 0;
};
#endif

#endif
