// Test infrastructure (oracle): drives the reference's OWN header-only hot-path physics on the CPU.
//
// The per-face functor FVM_Conservative2FluxHyperbolic_K, the surface integrals FVM_SurfaceIntegral /
// FVM_SurfaceIntegral_NC and the pressure relaxation Relaxation_Instantaneous are the reference's
// code, included from its include/ tree and compiled against oracle/refshim (an AMReX-compatible
// shim). Only the level-advance loop around them is restated here, following
//   ComputeFaceFluxes   source/Class_Compressible_PhaseField.cpp:3151-3254
//   FluxDivergence      source/Class_Compressible_PhaseField.cpp:3262-3391
//   ThirdOrderSSPRK     source/Class_Compressible_PhaseField.cpp:3937-4107
//   EstTimeStep         source/Class_Compressible_PhaseField.cpp:4472-4499
//   CalculateInitialcmax source/Class_Compressible_PhaseField.cpp:4501-4605
//   ComputeDt           source/COMPAS.cpp:2249-2303
//   Relaxation          source/Class_Compressible6Eq_PhaseField.cpp:46-59, 437-474
//   SetPhysicsBC        source/Class_Compressible6Eq_PhaseField.cpp:352-434 (5Eq: ...5Eq...:162-)
// One build per (PHYSICS, AMREX_SPACEDIM); see oracle/Makefile. Built into oracle/_ref only.
#include <AMReX.H>
#include <Macros.H>

// The reference's Tools.H aggregator pulls in output utilities; the physics needs only Sign.H.
#define Tools_H_
#include <Sign.H>

#include <Parm.H>

#if (PHYSICS == FIVEEQS_NPHASE)
#include <Physics_Compressible_NPhase.H>
#include <Physics_Compressible5Eq_NPhase.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
#include <Operators_Compressible5Eq_NPhase.H>
#elif (PHYSICS == SIXEQS_IE_NPHASE)
#include <Physics_Compressible_NPhase.H>
#include <Physics_Compressible6Eq_IE_NPhase.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
// the model's operator aggregator also pulls in its Phase-Field flux functor
#include <Physics_PhaseField.H>
#include <Physics_Compressible_NPhase_PhaseField.H>
#include <Physics_Compressible6Eq_IE_NPhase_PhaseField.H>
#include <Operators_Compressible6Eq_IE_NPhase.H>
#else
#include <Physics_Compressible_TwoPhase.H>
#endif
#if (PHYSICS == FIVEEQS)
#include <Physics_Compressible5Eq.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
#include <Operators_Compressible5Eq.H>
#include <Physics_PhaseField.H>
#include <Operators_PhaseField.H>
#include <Physics_Compressible_TwoPhase_PhaseField.H>
#include <Physics_Compressible5Eq_PhaseField.H>
#include <Operators_Compressible5Eq_PhaseField.H>
#elif (PHYSICS == SIXEQS)
#include <RelaxationPressure_Safeguarded.H>
#include <Physics_Compressible6Eq.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
#include <Operators_Compressible6Eq.H>
#include <Physics_PhaseField.H>
#include <Operators_PhaseField.H>
#include <Physics_Compressible_TwoPhase_PhaseField.H>
#include <Physics_Compressible6Eq_PhaseField.H>
#include <Operators_Compressible6Eq_PhaseField.H>
#endif

#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
// ErrorEst's tests (include/Tagging.H); its ProblemICBC.H is the shim's empty stand-in
#include <Tagging.H>
#endif

#include "oracle_api.h"

#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Geo {
    int nx, ny, nz, ng;
    int px, py, pz;
    long long S;
    int gz;  // ghosts in z (0 in 2D)
    Geo(const cmp_case* c) {
        nx = c->n[0];
        ny = c->n[1];
        nz = (AMREX_SPACEDIM == 3) ? c->n[2] : 1;
        ng = c->ng;
        gz = (AMREX_SPACEDIM == 3) ? ng : 0;
        px = nx + 2 * ng;
        py = ny + 2 * ng;
        pz = nz + 2 * gz;
        S = (long long)px * py * pz;
    }
    template <class T>
    amrex::Array4<T> view(T* p, int nc) const {
        return amrex::Array4<T>(p, amrex::Dim3{-ng, -ng, -gz}, amrex::Dim3{nx + ng, ny + ng, nz + gz}, nc);
    }
};

Parm make_parm(const cmp_case* c) {
    Parm p;
    p.EOS = 1;
#if (PHYSICS == FIVEEQS_NPHASE || PHYSICS == SIXEQS_IE_NPHASE)
    if (c->nphase != NPHASE) amrex::Abort("the case's nphase differs from this build's NPHASE");
    for (int k = 0; k < NPHASE; ++k) {
        p.A[k] = c->Ak[k]; p.B[k] = c->Bk[k]; p.C[k] = c->Ck[k]; p.D[k] = c->Dk[k];
        // source/Parm.cpp:255-261 (FIVEEQS_NPHASE), :446-450 (SIXEQS_IE_NPHASE: -B/(A + 1))
#if (PHYSICS == SIXEQS_IE_NPHASE)
        p.p_min[k] = -c->Bk[k] / (c->Ak[k] + 1.0);
        // the relaxation's NASG branch is taken for EOS = 3 with a covolume or heat of formation
        // (PressureRelaxation_IsNASG); the EOS 0 and 1 coefficients have C = D = 0
        if (c->Ck[k] > 0.0 || c->Dk[k] != 0.0) p.EOS = 3;
#else
        p.p_min[k] = (c->source_term == 1) ? -c->Bk[k] / (c->Ak[k] + 1.0) : -c->Bk[k] / c->Ak[k];
#endif
    }
#else
    p.A1 = c->A1; p.A2 = c->A2; p.B1 = c->B1; p.B2 = c->B2;
    p.C1 = c->C1; p.C2 = c->C2; p.D1 = c->D1; p.D2 = c->D2;
    // source/Parm.cpp:164-171
    if (c->source_term == 1) {
        p.p_min = {-c->B1 / (c->A1 + 1.0), -c->B2 / (c->A2 + 1.0)};
    } else {
        p.p_min = {-c->B1 / c->A1, -c->B2 / c->A2};
    }
#endif
    // FiniteVolume.Scheme (include/Operators_FV/FiniteVolume_Parameter.H:51-147)
    auto& fv = p.FiniteVolume_Parm;
    fv.ID_WENO = c->id_weno;
    fv.ID_Limiter = c->id_limiter;
    if (c->id_weno && (c->id_limiter == 3 || c->id_limiter == 4)) {
        fv.ID_Poly = 2;
        fv.Num_Grow = 2;
        fv.Scheme = (c->id_limiter == 4) ? FVReconstruction::WENO_3B : FVReconstruction::WENO_3;
    } else if (c->id_weno) {
        fv.ID_Poly = 4;
        fv.Num_Grow = 3;
        fv.Scheme = (c->id_limiter == 6) ? FVReconstruction::WENO_5B : FVReconstruction::WENO_5;
    } else {
        fv.ID_Poly = (c->id_limiter == 0) ? 0 : 1;
        fv.Num_Grow = (c->id_limiter == 0) ? 1 : 2;
        const FVReconstruction muscl[5] = {FVReconstruction::GODUNOV, FVReconstruction::MUSCL_MM,
                                           FVReconstruction::MUSCL_VL, FVReconstruction::MUSCL_SB,
                                           FVReconstruction::MUSCL_MC};
        fv.Scheme = muscl[c->id_limiter];
    }
    // FiniteVolume.ID_Bound: the MUSCL family runs its bounded form with ID_Poly 2 (:71-112); the
    // quadrature weight of the bounded branch's CFL speed follows ID_Poly (:161-173)
    fv.ID_Bound = c->id_bound;
    fv.ID_Lambda = c->id_lambda;
    if (c->id_bound && !c->id_weno && c->id_limiter > 0) fv.ID_Poly = 2;
    fv.Quadrature_Weight = (fv.ID_Poly == 0) ? 1.0 : (fv.ID_Poly == 1) ? 0.5 : (fv.ID_Poly == 2) ? 1.0 / 6.0 : 1.0 / 12.0;
    fv.ID_THINC = c->thinc;
    fv.ID_THINC_UseNormal = c->thinc_use_normal;
    fv.THINC_EPS = c->thinc_eps;
    fv.THINC_Beta = c->thinc_beta;
    fv.THINC_NormalThreshold = c->thinc_normal_threshold;
    p.Physics_Parm.ID_Riemann = c->id_riemann;
#if (PHYSICS == FIVEEQS || PHYSICS == FIVEEQS_NPHASE)
    p.Physics_Parm.source_term = c->source_term;
#elif (PHYSICS == SIXEQS)
    p.Physics_Parm.pressure_relaxation = c->relaxation;
    p.Physics_Parm.pressure_relaxation_trace = c->relax_trace;
    p.Physics_Parm.relaxation = c->relaxation;
#elif (PHYSICS == SIXEQS_IE_NPHASE)
    p.Physics_Parm.pressure_relaxation = c->relaxation;
    p.Physics_Parm.pressure_relaxation_trace = c->relax_trace;
#endif
    return p;
}

// AMReX BCType for component n in direction d at code `code`
// (source/Class_Compressible6Eq_PhaseField.cpp:362-431, Class_Compressible5Eq_NPhase_PhaseField.cpp:
// 133-205): 0 int_dir, 2 foextrap, 3/4 reflect_even (normal momentum reflect_odd), 5 reflect_odd for
// every momentum component.
enum { BC_INT = 0, BC_FOEXTRAP = 1, BC_EVEN = 2, BC_ODD = 3 };
int bc_kind(int code, int n, int d) {
#if (PHYSICS == FIVEEQS_NPHASE)
    const int m0 = NPHASE;
#elif (PHYSICS == SIXEQS_IE_NPHASE)
    const int m0 = 3 * NPHASE;
#else
    const int m0 = 2;
#endif
    const bool mom = (n >= m0 && n < m0 + AMREX_SPACEDIM);
    const bool normal = mom && (n - m0 == d);
    switch (code) {
        case 0: return BC_INT;
        case 2: return BC_FOEXTRAP;
        case 3:
        case 4: return normal ? BC_ODD : BC_EVEN;
        case 5: return mom ? BC_ODD : BC_EVEN;
        default: amrex::Abort("boundary code not supported by the oracle (inflow needs a user function)");
    }
}

void fill_ghosts(const cmp_case* c, double* U) {
    Geo g(c);
    const int nc = NSTATE;
    auto a = g.view(U, nc);
    const int lo[3] = {0, 0, 0};
    const int hi[3] = {g.nx - 1, g.ny - 1, g.nz - 1};
    const int ngd[3] = {g.ng, g.ng, g.gz};
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        for (int n = 0; n < nc; ++n) {
            for (int side = 0; side < 2; ++side) {
                const int code = side == 0 ? c->lo_bc[d] : c->hi_bc[d];
                const int kind = bc_kind(code, n, d);
                for (int k = -g.gz; k < g.nz + g.gz; ++k)
                for (int j = -g.ng; j < g.ny + g.ng; ++j)
                for (int i = -g.ng; i < g.nx + g.ng; ++i) {
                    int idx[3] = {i, j, k};
                    const int x = idx[d];
                    const bool ghost = side == 0 ? (x < lo[d]) : (x > hi[d]);
                    if (!ghost) continue;
                    // direction d only: the other directions keep their index
                    int src[3] = {i, j, k};
                    double sgn = 1.0;
                    const int len = hi[d] - lo[d] + 1;
                    if (kind == BC_INT) {
                        src[d] = side == 0 ? x + len : x - len;
                    } else if (kind == BC_FOEXTRAP) {
                        src[d] = side == 0 ? lo[d] : hi[d];
                    } else {
                        src[d] = side == 0 ? (2 * lo[d] - 1 - x) : (2 * hi[d] + 1 - x);
                        if (kind == BC_ODD) sgn = -1.0;
                    }
                    (void)ngd;
                    a(i, j, k, n) = sgn * a(src[0], src[1], src[2], n);
                }
            }
        }
    }
}

// ComputeFaceFluxes + FluxDivergence of one level state (ghosts filled). cmax: largest face wave
// speed over the faces (i,j,k) with (i,j,k) a valid cell (the low faces), as c_max.norminf(0,0,true).
void compute_dudt(const cmp_case* c, const Parm& parm, const double* U, double* dUdt, double* cmax_out,
                  std::vector<std::vector<double>>* faces_out = nullptr,
                  std::vector<std::vector<double>>* faces_nc_out = nullptr) {
    Geo g(c);
    const int nc = NSTATE;
    auto statein = g.view(U, nc);
    auto dudt = g.view(dUdt, nc);
    amrex::Array<amrex::Real, AMREX_SPACEDIM> dX = {AMREX_D_DECL(c->dx[0], c->dx[1], c->dx[2])};

    // face arrays: nodal in direction d, one extra layer
    std::vector<std::vector<double>> F(AMREX_SPACEDIM), FNC(AMREX_SPACEDIM);
    std::vector<amrex::Array4<double>> fa(AMREX_SPACEDIM), fnca(AMREX_SPACEDIM);
    double cmax_all = 0.0;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        int fx = g.nx + (d == 0), fy = g.ny + (d == 1), fz = g.nz + (d == 2);
        long long fs = (long long)fx * fy * fz;
        F[d].assign(fs * nc, 0.0);
        FNC[d].assign(fs * NC_TERMS, 0.0);
        fa[d] = amrex::Array4<double>(F[d].data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{fx, fy, fz}, nc);
        fnca[d] = amrex::Array4<double>(FNC[d].data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{fx, fy, fz}, NC_TERMS);
        double cm = 0.0;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) reduction(max : cm) schedule(static)
#endif
        for (int k = 0; k < fz; ++k)
        for (int j = 0; j < fy; ++j)
        for (int i = 0; i < fx; ++i) {
            amrex::Array<amrex::Real, NSTATE> fhat;
            amrex::Array<amrex::Real, NC_TERMS> fhatNC;
            amrex::Real cmax;
            FVM_Conservative2FluxHyperbolic_K(i, j, k, fhat, fhatNC, cmax, statein, parm, dX, d,
                                              parm.FiniteVolume_Parm, parm.Physics_Parm);
            for (int n = 0; n < nc; ++n) fa[d](i, j, k, n) = fhat[n];
            for (int n = 0; n < NC_TERMS; ++n) fnca[d](i, j, k, n) = fhatNC[n];
            const bool valid_low = (i < g.nx) && (j < g.ny) && (k < g.nz);
            if (valid_low) cm = std::max(cmax, cm);
        }
        cmax_all = std::max(cmax_all, cm);
    }
    amrex::Array4<amrex::Real const> fx_c = fa[0];
    amrex::Array4<amrex::Real const> fy_c = fa[1];
    amrex::Array4<amrex::Real const> fxnc_c = fnca[0];
    amrex::Array4<amrex::Real const> fync_c = fnca[1];
#if (AMREX_SPACEDIM == 3)
    amrex::Array4<amrex::Real const> fz_c = fa[2];
    amrex::Array4<amrex::Real const> fznc_c = fnca[2];
#endif
    const double dx = c->dx[0], dy = c->dx[1];
#if (AMREX_SPACEDIM == 3)
    const double dz = c->dx[2];
#endif
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
        for (int n = 0; n < nc; ++n) {
            FVM_SurfaceIntegral(i, j, k, n, dudt, statein,
                                AMREX_D_DECL(fx_c, fy_c, fz_c), AMREX_D_DECL(dx, dy, dz));
        }
        FVM_SurfaceIntegral_NC(i, j, k, dudt, statein,
                               AMREX_D_DECL(fx_c, fy_c, fz_c),
                               AMREX_D_DECL(fxnc_c, fync_c, fznc_c),
                               AMREX_D_DECL(dx, dy, dz), parm, parm.Physics_Parm);
    }
    if (cmax_out) *cmax_out = cmax_all;
    if (faces_out) *faces_out = F;
    if (faces_nc_out) *faces_nc_out = FNC;
}

void relax(const cmp_case* c, const Parm& parm, double* U) {
#if (PHYSICS == SIXEQS_IE_NPHASE)
    // PostTimeStage -> Relaxation_Pressure -> PressureRelaxationInstantaneous
    // (source/Class_Compressible6Eq_IE_NPhase_PhaseField.cpp:46-58, :464-472): the reference's cell
    // function on every valid cell, volume fractions and phase energies written back
    if (!parm.Physics_Parm.pressure_relaxation) return;
    const bool NASG = PressureRelaxation_IsNASG(parm);
    Geo g(c);
    auto a = g.view(U, NSTATE);
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
        amrex::Array<amrex::Real, NSTATE> Cons, ConsR;
        for (int n = 0; n < NSTATE; ++n) Cons[n] = a(i, j, k, n);
        int Iter, Path;
        PressureRelaxation_Cell(ConsR, Cons, parm, NASG, Iter, Path);
        for (int ph = 0; ph < NPHASE; ++ph) {
            a(i, j, k, INDEX_VolumeFraction1 + ph) = ConsR[INDEX_VolumeFraction1 + ph];
            a(i, j, k, INDEX_Energy1 + ph) = ConsR[INDEX_Energy1 + ph];
        }
    }
#elif (PHYSICS == SIXEQS)
    if (!parm.Physics_Parm.relaxation) return;
    Geo g(c);
    auto a = g.view(U, NSTATE);
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
        amrex::Array<amrex::Real, NSTATE> Cons, ConsR;
        for (int n = 0; n < NSTATE; ++n) Cons[n] = a(i, j, k, n);
        Relaxation_Instantaneous(ConsR, Cons, parm);
        for (int n = 0; n < NSTATE; ++n) a(i, j, k, n) = ConsR[n];
    }
#else
    (void)c; (void)parm; (void)U;
#endif
}

template <class F>
void for_valid(const Geo& g, F&& f) {
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int n = 0; n < NSTATE; ++n)
    for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j) {
        long long base = n * g.S + (long long)(k + g.gz) * g.py * g.px + (long long)(j + g.ng) * g.px + g.ng;
        for (int i = 0; i < g.nx; ++i) f(base + i);
    }
}

// MinEnergyBound (source/Class_Compressible_PhaseField.cpp:3596-3635): the smallest energy bound of the
// valid cells through the reference's Conservative2EnergyBound (AMReX's MultiFab::min restated as a
// running minimum; a NaN bound does not lower it). +inf for the models without the bounded branch.
double min_energy_bound(const cmp_case* c, const Parm& parm, const double* U) {
    double mn = std::numeric_limits<double>::infinity();
#if (PHYSICS == FIVEEQS || PHYSICS == FIVEEQS_NPHASE)
    Geo g(c);
    auto a = g.view(const_cast<double*>(U), NSTATE);
    for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
        amrex::Array<amrex::Real, NSTATE> Cons;
        for (int n = 0; n < NSTATE; ++n) Cons[n] = a(i, j, k, n);
        amrex::Real EB;
        Conservative2EnergyBound(EB, Cons, parm);
        if (EB < mn) mn = EB;
    }
#else
    (void)c; (void)parm; (void)U;
#endif
    return mn;
}

// The energy check after a stage of ThirdOrderSSPRK under ID_Bound = 1 (:4014-4030): true when the
// step has to be taken again.
bool bound_violated(const cmp_case* c, const Parm& parm, const double* U) {
    return parm.FiniteVolume_Parm.ID_Bound == 1 && min_energy_bound(c, parm, U) < 0;
}

int g_bound_restarts = 0;

// ThirdOrderSSPRK: the stage combinations as MultiFab::LinComb / Saxpy compute them
// (dst = a*x + b*y, then dst += a*x), with PostTimeStage (relaxation) after each stage. Returns 1
// (U holding the violating stage state) when an energy check fails, 0 otherwise.
int rk3_step(const cmp_case* c, const Parm& parm, double* U, double dt, double* cmax_out) {
    Geo g(c);
    const long long tot = g.S * NSTATE;
    std::vector<double> U0(U, U + tot), Ub(tot), L(tot, 0.0);
    double cm = 0.0, cms = 0.0;
    // stage 1
    std::memcpy(Ub.data(), U0.data(), tot * sizeof(double));
    fill_ghosts(c, Ub.data());
    compute_dudt(c, parm, Ub.data(), L.data(), &cms);
    cm = std::max(cm, cms);
    for_valid(g, [&](long long q) { U[q] = 1.0 * Ub[q] + dt * L[q]; });
    relax(c, parm, U);
    if (bound_violated(c, parm, U)) return 1;
    // stage 2
    std::memcpy(Ub.data(), U, tot * sizeof(double));
    fill_ghosts(c, Ub.data());
    compute_dudt(c, parm, Ub.data(), L.data(), &cms);
    cm = std::max(cm, cms);
    const double s2 = 0.25 * dt;
    for_valid(g, [&](long long q) {
        U[q] = 0.25 * Ub[q] + 0.75 * U0[q];
        U[q] += s2 * L[q];
    });
    relax(c, parm, U);
    if (bound_violated(c, parm, U)) return 1;
    // stage 3
    std::memcpy(Ub.data(), U, tot * sizeof(double));
    fill_ghosts(c, Ub.data());
    compute_dudt(c, parm, Ub.data(), L.data(), &cms);
    cm = std::max(cm, cms);
    const double a3 = 2.0 / 3.0, b3 = 1.0 / 3.0, s3 = (2.0 / 3.0) * dt;
    for_valid(g, [&](long long q) {
        U[q] = a3 * Ub[q] + b3 * U0[q];
        U[q] += s3 * L[q];
    });
    relax(c, parm, U);
    if (bound_violated(c, parm, U)) return 1;
    if (cmax_out) *cmax_out = cm;
    return 0;
}

double est_dt(const cmp_case* c, double cmax) {
    double dt = std::numeric_limits<double>::max();
    for (int d = 0; d < AMREX_SPACEDIM; ++d) dt = amrex::min(dt, c->cfl * c->dx[d] / cmax);
    return dt;
}

#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
// ------------------------------------------------------------------------------------------------
// Phase-Field regularisation step (FIVEEQS and SIXEQS, NPHASE = 1), restating the orchestration of
//   PhaseField_Evolve              source/Class_Compressible_PhaseField.cpp:424-595
//   PhaseFieldMechanism_Evolve     :596-711
//   PhaseField_Mechanism (CAC)     :1006-1152, (flux-based) :1155-1232, PhaseField_ACDI :1494-1645
//   PhaseField_Normal              :1957-2033
//   PhaseField_GradQPF (implicit)  :2132-2310, (explicit) :2314-2401
//   PhaseField_ComputeDt           :2036-2098
//   PhaseField_ThirdOrderSSPRK     :2619-2752, PhaseField_ComputeFaceFluxes :770-855,
//   PhaseField_FluxDivergence      :858-947
// around the reference's own device functions. AMReX pieces restated from their documented
// semantics: FillPatch of the phase field and of the normals (int_dir on periodic directions,
// foextrap elsewhere), MultiFab::sum / norminf, and the MLMG solve of the ABecLaplacian
// (a = 0, b = -1: div(beta grad Q) = rhs; singular with Neumann / periodic sides, made solvable by
// removing the mean of rhs), here a conjugate-gradient solve to a tight tolerance.
// ------------------------------------------------------------------------------------------------

// Padded scalar (nc components) field with g ghost cells (none in z in 2D).
struct SField {
    int nx, ny, nz, g, gz, nc;
    std::vector<double> v;
    SField(const Geo& G, int ng, int ncomp) : nx(G.nx), ny(G.ny), nz(G.nz), g(ng), gz(AMREX_SPACEDIM == 3 ? ng : 0), nc(ncomp) {
        v.assign((size_t)(nx + 2 * g) * (ny + 2 * g) * (nz + 2 * gz) * nc, 0.0);
    }
    amrex::Array4<double> a() { return amrex::Array4<double>(v.data(), amrex::Dim3{-g, -g, -gz}, amrex::Dim3{nx + g, ny + g, nz + gz}, nc); }
};

// Face field of direction d (nodal in d, no ghosts).
struct FField {
    int fx, fy, fz;
    std::vector<double> v;
    FField() : fx(0), fy(0), fz(0) {}
    FField(const Geo& G, int d) : fx(G.nx + (d == 0)), fy(G.ny + (d == 1)), fz(G.nz + (d == 2)) {
        v.assign((size_t)fx * fy * fz, 0.0);
    }
    amrex::Array4<double> a() { return amrex::Array4<double>(v.data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{fx, fy, fz}, 1); }
};

// FillPatch with PF_bcs / Normal_bcs: int_dir on periodic directions, foextrap elsewhere, direction by
// direction over the full extent of the others.
void fill_pf(const cmp_case* c, SField& f) {
    auto a = f.a();
    const int n[3] = {f.nx, f.ny, f.nz};
    const int gg[3] = {f.g, f.g, f.gz};
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
        for (int comp = 0; comp < f.nc; ++comp)
            for (int k = -f.gz; k < f.nz + f.gz; ++k)
                for (int j = -f.g; j < f.ny + f.g; ++j)
                    for (int i = -f.g; i < f.nx + f.g; ++i) {
                        int idx[3] = {i, j, k};
                        const int x = idx[d];
                        if (x >= 0 && x < n[d]) continue;
                        int src[3] = {i, j, k};
                        if (c->lo_bc[d] == 0) src[d] = (x < 0) ? x + n[d] : x - n[d];
                        else src[d] = (x < 0) ? 0 : n[d] - 1;
                        a(i, j, k, comp) = a(src[0], src[1], src[2], comp);
                    }
    (void)gg;
}

template <class F>
void cells(const Geo& g, F&& f) {
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) f(i, j, k);
}

template <class F>
void faces(const Geo& g, int d, F&& f) {
    for (int k = 0; k < g.nz + (d == 2); ++k)
        for (int j = 0; j < g.ny + (d == 1); ++j)
            for (int i = 0; i < g.nx + (d == 0); ++i) f(i, j, k);
}

struct PfSetup {
    PhaseField_Parameter P;  // Lambda, Eta, Mobility as PhaseField_Evolve sets them
    double max_v;
};

// MaxVelocity (:3540-3577) and the parameter defaults of PhaseField_Evolve (:426-463).
PfSetup pf_setup(const cmp_case* c, const cmp_pf* pf, const double* U) {
    Geo g(c);
    auto st = g.view(const_cast<double*>(U), NSTATE);
    double vmax = 0.0;
    cells(g, [&](int i, int j, int k) {
        amrex::Array<amrex::Real, NSTATE> C;
        for (int n = 0; n < NSTATE; ++n) C[n] = st(i, j, k, n);
        AMREX_D_TERM(amrex::Real u;, amrex::Real v;, amrex::Real w);
        Conservative2Velocity(AMREX_D_DECL(u, v, w), C);
        const double V = std::sqrt(AMREX_D_TERM(u * u, +v * v, +w * w));
        vmax = std::max(vmax, std::abs(V));
    });
    PfSetup s;
    s.max_v = vmax;
    s.P.Lambda = pf->lambda;
    if (s.P.Lambda <= 0.0) s.P.Lambda = 1.0;
    s.P.Eta = pf->eta;
    if (s.P.Eta <= 0.0) {
        double dxm = c->dx[0];
        for (int d = 1; d < AMREX_SPACEDIM; ++d) dxm = std::max(dxm, c->dx[d]);
        s.P.Eta = pf->eta_multiplier * dxm;
    }
    s.P.Eta_Factor = pf->eta_factor;
    s.P.Mobility = 1.0;
    s.P.Mobility *= 0.5 * s.P.Eta * vmax;  // non-CH mechanisms
    s.P.ID_Mechanism = pf->mechanism;
    s.P.ID_ExplicitRC = pf->explicit_rc;
    s.P.ID_FluxPhase2Flux = pf->phase2flux;
    s.P.ID_Flux = pf->flux;
    s.P.cfl = pf->cfl;
    s.P.max_step = pf->max_step;
    return s;
}

// PhaseField_Normal: unit normal of field f (component 0) at the valid cells, then NormalBorder with
// one ghost layer.
void pf_normal(const cmp_case* c, SField& f, SField& nrm) {
    Geo g(c);
    auto fa = f.a();
    auto na = nrm.a();
    const double dx = c->dx[0], dy = c->dx[1];
#if (AMREX_SPACEDIM == 3)
    const double dz = c->dx[2];
#endif
    amrex::Array4<amrex::Real const> fc = fa;
    cells(g, [&](int i, int j, int k) {
        amrex::Array<amrex::Real, AMREX_SPACEDIM> Nf;
        FDM_Normal_CenterFromCenter_K(i, j, k, 0, Nf, fc, AMREX_D_DECL(dx, dy, dz));
        for (int d = 0; d < AMREX_SPACEDIM; ++d) na(i, j, k, d) = Nf[d];
    });
    fill_pf(c, nrm);
}

// Div_J of the CAC mechanism (ID_Mechanism 1, FDM_PhaseFieldMechanism_ACAdv_K) for PFBorder pfb.
void pf_mechanism_cac(const cmp_case* c, const PhaseField_Parameter& P, SField& pfb, std::vector<double>& divj) {
    Geo g(c);
    SField nrm(g, 1, AMREX_SPACEDIM);
    pf_normal(c, pfb, nrm);
    SField mob(g, 0, 1);
    std::fill(mob.v.begin(), mob.v.end(), P.Mobility);
    amrex::Array4<amrex::Real const> pa = pfb.a(), na = nrm.a(), ma = mob.a();
    const double dx = c->dx[0], dy = c->dx[1];
#if (AMREX_SPACEDIM == 3)
    const double dz = c->dx[2];
#endif
    const size_t nv = (size_t)g.nx * g.ny * g.nz;
    std::vector<double> mech(nv), wgt(nv);
    size_t q = 0;
    cells(g, [&](int i, int j, int k) {
        amrex::Real m;
        FDM_PhaseFieldMechanism_ACAdv_K(i, j, k, 0, m, pa, na, ma, P.Lambda, P.Eta, AMREX_D_DECL(dx, dy, dz),
                                        P.ID_Potential);
        amrex::Real w;
        WeightFunction_PhaseField(w, pa(i, j, k, 0), 0, P.ID_Weight);
        mech[q] = m;
        wgt[q] = w;
        ++q;
    });
    double im = 0.0, iw = 0.0;
    for (size_t t = 0; t < nv; ++t) {
        im += mech[t];
        iw += wgt[t];
    }
    divj.resize(nv);
    for (size_t t = 0; t < nv; ++t) {
        amrex::Real out;
        PhaseFieldMechanism_CAC(out, mech[t], im, wgt[t], iw);
        divj[t] = out;
    }
}

// J_Flux of the ACDI mechanism (ID_Mechanism 3) on the faces, and Div_J.
void pf_mechanism_acdi(const cmp_case* c, const PhaseField_Parameter& P, SField& pfb, std::vector<FField>& J,
                       std::vector<double>& divj) {
    Geo g(c);
    SField ls(g, 1, 1);
    auto la = ls.a();
    auto pa = pfb.a();
    cells(g, [&](int i, int j, int k) {
        amrex::Real l;
        Mapping_Backward(l, pa(i, j, k, 0), P.Eta, 0);
        la(i, j, k, 0) = l;
    });
    fill_pf(c, ls);
    SField nrm(g, 1, AMREX_SPACEDIM);
    pf_normal(c, ls, nrm);
    SField mob(g, 1, 1);
    std::fill(mob.v.begin(), mob.v.end(), P.Mobility);
    amrex::Array4<amrex::Real const> pc = pa, nc = nrm.a(), mc = mob.a();
    J.assign(AMREX_SPACEDIM, FField());
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        J[d] = FField(g, d);
        auto ja = J[d].a();
        faces(g, d, [&](int i, int j, int k) {
            amrex::Real fl;
            FDM_PhaseFieldFlux_ACDI_K(i, j, k, 0, fl, pc, nc, mc, P.Eta, c->dx[d], d);
            ja(i, j, k, 0) = fl;
        });
    }
    divj.assign((size_t)g.nx * g.ny * g.nz, 0.0);
    amrex::Array4<amrex::Real const> jx = J[0].a(), jy = J[1].a();
#if (AMREX_SPACEDIM == 3)
    amrex::Array4<amrex::Real const> jz = J[2].a();
#endif
    const double dx = c->dx[0], dy = c->dx[1];
#if (AMREX_SPACEDIM == 3)
    const double dz = c->dx[2];
#endif
    size_t q = 0;
    cells(g, [&](int i, int j, int k) {
        amrex::Real dv;
        FVM_Divergence_K(i, j, k, 0, dv, AMREX_D_DECL(jx, jy, jz), AMREX_D_DECL(dx, dy, dz));
        divj[q++] = dv;
    });
}

// Face value of the mapped phase field (Mapping_Backward with Eta, Mapping_Forward with
// Eta_Factor * Eta, linear face average), as the two PhaseField_GradQPF variants compute it.
double pf_face_mapped(double pc, double pm, const PhaseField_Parameter& P) {
    amrex::Real psic, psim, fc, fm, face;
    Mapping_Backward(psic, pc, P.Eta, 0);
    Mapping_Backward(psim, pm, P.Eta, 0);
    Mapping_Forward(fc, psic, P.Eta_Factor * P.Eta, 0);
    Mapping_Forward(fm, psim, P.Eta_Factor * P.Eta, 0);
    Interpolation2Face_Linear_D(face, fm, fc);
    return face;
}

// Conjugate-gradient solve of div(beta grad Q) = rhs on the valid cells with homogeneous Neumann
// (non-periodic) or periodic sides; rhs has its mean removed first (singular operator).
void pf_solve(const cmp_case* c, const std::vector<FField>& beta, std::vector<double> rhs, std::vector<double>& Q,
              double tol) {
    Geo g(c);
    const int n[3] = {g.nx, g.ny, g.nz};
    const size_t nv = (size_t)g.nx * g.ny * g.nz;
    auto id = [&](int i, int j, int k) { return (size_t)i + (size_t)g.nx * ((size_t)j + (size_t)g.ny * k); };
    double mean = 0.0;
    for (double r : rhs) mean += r;
    mean /= (double)nv;
    for (double& r : rhs) r -= mean;
    // A x = -div(beta grad x) (symmetric positive semi-definite)
    auto apply = [&](const std::vector<double>& x, std::vector<double>& y) {
        for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
                for (int i = 0; i < g.nx; ++i) {
                    const int ci[3] = {i, j, k};
                    double acc = 0.0;
                    const double xc = x[id(i, j, k)];
                    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
                        const double h2 = c->dx[d] * c->dx[d];
                        for (int s = 0; s < 2; ++s) {
                            int nb[3] = {ci[0], ci[1], ci[2]};
                            nb[d] += s ? 1 : -1;
                            const bool out = nb[d] < 0 || nb[d] >= n[d];
                            if (out && c->lo_bc[d] != 0) continue;  // Neumann: no flux through the side
                            if (out) nb[d] = (nb[d] + n[d]) % n[d];
                            int fi[3] = {ci[0], ci[1], ci[2]};
                            if (s) fi[d] += 1;
                            const FField& b = beta[d];
                            const double bf = b.v[(size_t)fi[0] + (size_t)b.fx * ((size_t)fi[1] + (size_t)b.fy * fi[2])];
                            acc += bf * (xc - x[id(nb[0], nb[1], nb[2])]) / h2;
                        }
                    }
                    y[id(i, j, k)] = acc;
                }
    };
    std::vector<double> x(nv, 0.0), r(nv), z(nv), p(nv), Ap(nv), diag(nv, 0.0);
    for (size_t t = 0; t < nv; ++t) r[t] = -rhs[t];
    // Jacobi preconditioner
    {
        std::vector<double> e(nv, 0.0), ae(nv);
        for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
                for (int i = 0; i < g.nx; ++i) {
                    double dsum = 0.0;
                    const int ci[3] = {i, j, k};
                    for (int d = 0; d < AMREX_SPACEDIM; ++d)
                        for (int s = 0; s < 2; ++s) {
                            int nb = ci[d] + (s ? 1 : -1);
                            if ((nb < 0 || nb >= n[d]) && c->lo_bc[d] != 0) continue;
                            int fi[3] = {ci[0], ci[1], ci[2]};
                            if (s) fi[d] += 1;
                            const FField& b = beta[d];
                            dsum += b.v[(size_t)fi[0] + (size_t)b.fx * ((size_t)fi[1] + (size_t)b.fy * fi[2])] / (c->dx[d] * c->dx[d]);
                        }
                    diag[id(i, j, k)] = dsum;
                }
    }
    auto precond = [&](const std::vector<double>& in, std::vector<double>& out) {
        double m = 0.0;
        for (size_t t = 0; t < nv; ++t) {
            out[t] = diag[t] > 0.0 ? in[t] / diag[t] : in[t];
            m += out[t];
        }
        m /= (double)nv;
        for (size_t t = 0; t < nv; ++t) out[t] -= m;
    };
    double rn0 = 0.0;
    for (double v : r) rn0 = std::max(rn0, std::abs(v));
    precond(r, z);
    p = z;
    double rz = 0.0;
    for (size_t t = 0; t < nv; ++t) rz += r[t] * z[t];
    for (int it = 0; it < 100000 && rn0 > 0.0; ++it) {
        apply(p, Ap);
        double pAp = 0.0;
        for (size_t t = 0; t < nv; ++t) pAp += p[t] * Ap[t];
        if (!(pAp > 0.0)) break;
        const double al = rz / pAp;
        double rn = 0.0;
        for (size_t t = 0; t < nv; ++t) {
            x[t] += al * p[t];
            r[t] -= al * Ap[t];
            rn = std::max(rn, std::abs(r[t]));
        }
        if (rn <= tol * rn0) break;
        precond(r, z);
        double rz2 = 0.0;
        for (size_t t = 0; t < nv; ++t) rz2 += r[t] * z[t];
        const double be = rz2 / rz;
        rz = rz2;
        for (size_t t = 0; t < nv; ++t) p[t] = z[t] + be * p[t];
    }
    Q = x;
}

// Grad_QPF on the faces for the state U (PhaseField_Evolve up to the Phase-Field time loop).
void pf_grad_q(const cmp_case* c, const cmp_pf* pf, const PfSetup& S, const double* U, double dt,
               std::vector<FField>& GQ, double* info) {
    Geo g(c);
    const PhaseField_Parameter& P = S.P;
    const size_t nv = (size_t)g.nx * g.ny * g.nz;
    auto st = g.view(const_cast<double*>(U), NSTATE);
    // PFBorder from the state (NGROW ghosts)
    SField pfb0(g, c->ng, 1);
    {
        auto a = pfb0.a();
        cells(g, [&](int i, int j, int k) { a(i, j, k, 0) = st(i, j, k, INDEX_VolumeFraction1); });
        fill_pf(c, pfb0);
    }
    // PhaseFieldMechanism_Evolve
    std::vector<double> pf0(nv), pfn(nv), pfo(nv);
    {
        size_t q = 0;
        auto a = pfb0.a();
        cells(g, [&](int i, int j, int k) { pf0[q++] = a(i, j, k, 0); });
    }
    pfn = pf0;
    double dxm[3] = {c->dx[0], c->dx[1], AMREX_SPACEDIM == 3 ? c->dx[2] : 1.0};
    double mdt = 0.9 / (2.0 * P.Mobility * P.Lambda) /
                 (AMREX_D_TERM(1.0 / dxm[0] / dxm[0], +1.0 / dxm[1] / dxm[1], +1.0 / dxm[2] / dxm[2]) + 1.0 / P.Eta / P.Eta);
    double mt = 0.0;
    const double T = dt;
    int msteps = 0;
    std::vector<FField> Jhat(AMREX_SPACEDIM);
    for (int d = 0; d < AMREX_SPACEDIM; ++d) Jhat[d] = FField(g, d);
    while (mt < T) {
        if (mt + mdt > T) mdt = T - mt;
        pfo = pfn;
        SField pfb(g, c->ng, 1);
        {
            auto a = pfb.a();
            size_t q = 0;
            cells(g, [&](int i, int j, int k) { a(i, j, k, 0) = pfn[q++]; });
            fill_pf(c, pfb);
        }
        std::vector<double> divj;
        if (pf->mechanism == 1) {
            pf_mechanism_cac(c, P, pfb, divj);
        } else {
            std::vector<FField> J;
            pf_mechanism_acdi(c, P, pfb, J, divj);
            if (P.ID_ExplicitRC == 1)
                for (int d = 0; d < AMREX_SPACEDIM; ++d)
                    for (size_t t = 0; t < Jhat[d].v.size(); ++t) Jhat[d].v[t] += mdt * J[d].v[t];
        }
        for (size_t t = 0; t < nv; ++t) pfn[t] = 1.0 * pfo[t] + mdt * divj[t];
        mt += mdt;
        ++msteps;
    }
    GQ.assign(AMREX_SPACEDIM, FField());
    for (int d = 0; d < AMREX_SPACEDIM; ++d) GQ[d] = FField(g, d);
    auto pa = pfb0.a();
    if (P.ID_ExplicitRC == 1) {
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
            for (double& v : Jhat[d].v) v *= (1.0 / dt);
            auto ja = Jhat[d].a();
            auto ga = GQ[d].a();
            faces(g, d, [&](int i, int j, int k) {
                const double pm = pa(i - (d == 0), j - (d == 1), k - (d == 2), 0);
                const double face = pf_face_mapped(pa(i, j, k, 0), pm, P);
                amrex::Real gq;
                PhaseFieldFlux2GradQPF(gq, ja(i, j, k, 0), face, 1.0e-3);
                ga(i, j, k, 0) = gq;
            });
        }
    } else {
        std::vector<double> djhat(nv);
        for (size_t t = 0; t < nv; ++t) djhat[t] = (1.0 / dt) * pfn[t] + (-1.0 / dt) * pf0[t];
        std::vector<FField> beta(AMREX_SPACEDIM);
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
            beta[d] = FField(g, d);
            auto ba = beta[d].a();
            faces(g, d, [&](int i, int j, int k) {
                const double pm = pa(i - (d == 0), j - (d == 1), k - (d == 2), 0);
                const double face = pf_face_mapped(pa(i, j, k, 0), pm, P);
                amrex::Real w;
                WeightFunction_PhaseField(w, face, 0, P.ID_Weight);
                ba(i, j, k, 0) = w + 1.0e-3;
            });
        }
        std::vector<double> Q;
        pf_solve(c, beta, djhat, Q, pf->tol_rel);
        const int n[3] = {g.nx, g.ny, g.nz};
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
            auto ga = GQ[d].a();
            faces(g, d, [&](int i, int j, int k) {
                int ci[3] = {i, j, k};
                int mi[3] = {i, j, k};
                mi[d] -= 1;
                double val;
                if (ci[d] == 0 || ci[d] == n[d]) {
                    if (c->lo_bc[d] != 0) {
                        ga(i, j, k, 0) = 0.0;  // homogeneous Neumann
                        return;
                    }
                    ci[d] = (ci[d] + n[d]) % n[d];
                    mi[d] = (mi[d] + n[d]) % n[d];
                }
                const size_t qc = (size_t)ci[0] + (size_t)g.nx * ((size_t)ci[1] + (size_t)g.ny * ci[2]);
                const size_t qm = (size_t)mi[0] + (size_t)g.nx * ((size_t)mi[1] + (size_t)g.ny * mi[2]);
                val = (Q[qc] - Q[qm]) / c->dx[d];
                ga(i, j, k, 0) = val;
            });
        }
    }
    if (info) {
        double gmax = 0.0;
        for (int d = 0; d < AMREX_SPACEDIM; ++d)
            for (double v : GQ[d].v) gmax = std::max(gmax, std::abs(v));
        info[0] = S.max_v;
        info[1] = P.Mobility;
        info[2] = P.Eta;
        info[3] = msteps;
        info[5] = gmax;
    }
}

// PhaseField_compute_dUdt_FV of a state with filled ghosts (PhaseField_ComputeFaceFluxes :770-855 and
// PhaseField_FluxDivergence :858-947): fluxes -fhat and the non-conservative terms +fhatNC on the faces,
// the surface integral, then PhaseField_FVM_SurfaceIntegral_NC (empty for FIVEEQS; the phase-energy
// exchange for SIXEQS).
void pf_compute_dudt(const cmp_case* c, const Parm& parm, const double* Ub, const std::vector<FField>& GQ,
                     double* dUdt) {
    Geo g(c);
    auto statein = g.view(const_cast<double*>(Ub), NSTATE);
    auto dudt = g.view(dUdt, NSTATE);
    std::vector<std::vector<double>> F(AMREX_SPACEDIM), FNC(AMREX_SPACEDIM);
    std::vector<amrex::Array4<double>> fa(AMREX_SPACEDIM), fnca(AMREX_SPACEDIM);
    amrex::Array4<amrex::Real const> sc = statein;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        const int fx = g.nx + (d == 0), fy = g.ny + (d == 1), fz = g.nz + (d == 2);
        F[d].assign((size_t)fx * fy * fz * NSTATE, 0.0);
        fa[d] = amrex::Array4<double>(F[d].data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{fx, fy, fz}, NSTATE);
        FNC[d].assign((size_t)fx * fy * fz * NC_TERMS, 0.0);
        fnca[d] = amrex::Array4<double>(FNC[d].data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{fx, fy, fz}, NC_TERMS);
        const FField& gq = GQ[d];
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
        for (int k = 0; k < fz; ++k)
            for (int j = 0; j < fy; ++j)
                for (int i = 0; i < fx; ++i) {
                    amrex::Array<amrex::Real, NPHASE> grad;
                    grad[0] = gq.v[(size_t)i + (size_t)fx * ((size_t)j + (size_t)fy * k)];
                    amrex::Array<amrex::Real, NSTATE> fhat;
                    amrex::Array<amrex::Real, NC_TERMS> fhatNC;
                    amrex::Real cmax;
                    FVM_Conservative2FluxPhaseField_K(i, j, k, fhat, fhatNC, cmax, sc, grad, parm, c->dx[d], d,
                                                      parm.FiniteVolume_Parm, parm.PhaseField_Parm);
                    for (int n = 0; n < NSTATE; ++n) fa[d](i, j, k, n) = -fhat[n];
                    for (int n = 0; n < NC_TERMS; ++n) fnca[d](i, j, k, n) = fhatNC[n];
                }
    }
    amrex::Array4<amrex::Real const> fx_c = fa[0], fy_c = fa[1];
    amrex::Array4<amrex::Real const> fxnc_c = fnca[0], fync_c = fnca[1];
#if (AMREX_SPACEDIM == 3)
    amrex::Array4<amrex::Real const> fz_c = fa[2];
    amrex::Array4<amrex::Real const> fznc_c = fnca[2];
#endif
    const double dx = c->dx[0], dy = c->dx[1];
#if (AMREX_SPACEDIM == 3)
    const double dz = c->dx[2];
#endif
    cells(g, [&](int i, int j, int k) {
        for (int n = 0; n < NSTATE; ++n)
            FVM_SurfaceIntegral(i, j, k, n, dudt, statein, AMREX_D_DECL(fx_c, fy_c, fz_c), AMREX_D_DECL(dx, dy, dz));
        PhaseField_FVM_SurfaceIntegral_NC(i, j, k, dudt, statein, AMREX_D_DECL(fxnc_c, fync_c, fznc_c),
                                          AMREX_D_DECL(dx, dy, dz), parm);
    });
}

// The sub-stepped Phase-Field TVD-RK3 advance over dt with fixed face gradients.
int pf_advance(const cmp_case* c, const cmp_pf* pf, const PfSetup& S, double* U, double dt, const std::vector<FField>& GQ,
               double gmax) {
    Geo g(c);
    Parm parm = make_parm(c);
    parm.PhaseField_Parm = S.P;
    double dxmin = c->dx[0];
    for (int d = 1; d < AMREX_SPACEDIM; ++d) dxmin = std::min(dxmin, c->dx[d]);
    const long long tot = g.S * NSTATE;
    double pft = 0.0, pfdt = 0.0;
    int steps = 0;
    for (int s = 0; s < S.P.max_step && pft < dt; ++s) {
        // PhaseField_ComputeDt
        double tmp = S.P.cfl * dxmin / (gmax + 1.0e-14);
        if (pft == 0.0) pfdt = tmp;
        if (c->change_limiter && pfdt > 0.0) tmp = std::min(tmp, 1.1 * pfdt);
        double d0 = tmp;
        const double eps = 1.0e-3 * d0;
        if (pft + d0 > dt - eps) d0 = dt - pft;
        pfdt = d0;
        // PhaseField_ThirdOrderSSPRK
        std::vector<double> U0(U, U + tot), Ub(tot), L(tot, 0.0);
        std::memcpy(Ub.data(), U0.data(), tot * sizeof(double));
        fill_ghosts(c, Ub.data());
        pf_compute_dudt(c, parm, Ub.data(), GQ, L.data());
        for_valid(g, [&](long long q) { U[q] = 1.0 * Ub[q] + pfdt * L[q]; });
        relax(c, parm, U);  // PhaseField_PostTimeStage (SIXEQS: Relaxation; nothing for FIVEEQS)
        std::memcpy(Ub.data(), U, tot * sizeof(double));
        fill_ghosts(c, Ub.data());
        pf_compute_dudt(c, parm, Ub.data(), GQ, L.data());
        const double s2 = 0.25 * pfdt;
        for_valid(g, [&](long long q) {
            U[q] = 0.25 * Ub[q] + 0.75 * U0[q];
            U[q] += s2 * L[q];
        });
        relax(c, parm, U);
        std::memcpy(Ub.data(), U, tot * sizeof(double));
        fill_ghosts(c, Ub.data());
        pf_compute_dudt(c, parm, Ub.data(), GQ, L.data());
        const double a3 = 2.0 / 3.0, b3 = 1.0 / 3.0, s3 = (2.0 / 3.0) * pfdt;
        for_valid(g, [&](long long q) {
            U[q] = a3 * Ub[q] + b3 * U0[q];
            U[q] += s3 * L[q];
        });
        relax(c, parm, U);
        pft += pfdt;
        ++steps;
        if (pft >= dt - 1.0e-6 * dt) break;
    }
    return steps;
}

void pf_step(const cmp_case* c, const cmp_pf* pf, double* U, double dt, double* info) {
    PfSetup S = pf_setup(c, pf, U);
    std::vector<FField> GQ;
    double loc[6] = {0, 0, 0, 0, 0, 0};
    pf_grad_q(c, pf, S, U, dt, GQ, loc);
    loc[4] = pf_advance(c, pf, S, U, dt, GQ, loc[5]);
    if (info)
        for (int t = 0; t < 6; ++t) info[t] = loc[t];
}
#endif  // PHYSICS == FIVEEQS || PHYSICS == SIXEQS

#include "ref_amr.inc"

template <class Fn>
int guarded(Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle (reference build): %s\n", e.what());
        return -1;
    }
}

}  // namespace

extern "C" {

int cmp_nstate(const cmp_case*) { return NSTATE; }

int cmp_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int cmp_fill_ghosts(const cmp_case* c, double* U) {
    return guarded([&] { fill_ghosts(c, U); });
}

int cmp_compute_dudt(const cmp_case* c, const double* U, double* dUdt, double* cmax) {
    return guarded([&] {
        Parm parm = make_parm(c);
        compute_dudt(c, parm, U, dUdt, cmax);
    });
}

int cmp_relax(const cmp_case* c, double* U) {
    return guarded([&] {
        Parm parm = make_parm(c);
        relax(c, parm, U);
    });
}

int cmp_rk3_step(const cmp_case* c, double* U, double dt, double* cmax) {
    int violated = 0;
    const int rc = guarded([&] {
        Parm parm = make_parm(c);
        violated = rk3_step(c, parm, U, dt, cmax);
    });
    return rc ? rc : violated;
}

int cmp_energy_bound_min(const cmp_case* c, const double* U, double* out) {
    return guarded([&] {
        Parm parm = make_parm(c);
        *out = min_energy_bound(c, parm, U);
    });
}

int cmp_bound_restarts(void) { return g_bound_restarts; }

int cmp_advance(const cmp_case* c, double* U, int nsteps, double stop_time, double* t, double* dts) {
    int taken = 0;
    g_bound_restarts = 0;
    int rc = guarded([&] {
        Parm parm = make_parm(c);
        parm.FiniteVolume_Parm.ID_Lambda = 1;  // the struct default; the step taken again switches it
        Geo g(c);
        const long long tot = g.S * NSTATE;
        double dt_prev = 1.e100;  // COMPAS::dt starts at 1e100 (source/COMPAS.cpp:81)
        double cmax = 0.0;
        double time = *t;
        for (int step = 0; step < nsteps && time < stop_time; ++step) {
            if (time == 0.0) {
                // CalculateInitialcmax: the face speeds of the state at t = 0
                std::vector<double> Ub(U, U + g.S * NSTATE), L(g.S * NSTATE);
                fill_ghosts(c, Ub.data());
                compute_dudt(c, parm, Ub.data(), L.data(), &cmax);
            }
            double dt_est = est_dt(c, cmax);
            if (time == 0.0) dt_prev = dt_est;
            if (c->change_limiter && dt_prev > 0.0) dt_est = std::min(dt_est, 1.1 * dt_prev);
            double dt0 = dt_est;
            const double eps = 1.0e-3 * dt0;
            if (time + dt0 > stop_time - eps) dt0 = stop_time - time;
            dt_prev = dt0;
            std::vector<double> Usave;
            if (parm.FiniteVolume_Parm.ID_Bound == 1) Usave.assign(U, U + tot);
            if (rk3_step(c, parm, U, dt0, &cmax)) {
                // Evolve under ID_Bound = 1 (source/Class_Compressible_PhaseField.cpp:264-306):
                // RemakeAllLevelsFromData back to the state the step started from, ID_Lambda = 0,
                // ComputeDt with ID_Return = 1 (CalculateInitialcmax of that state, :4481-4483; the
                // change limiter against the failed dt), the step again, ID_Lambda = 1
                ++g_bound_restarts;
                std::memcpy(U, Usave.data(), sizeof(double) * tot);
                parm.FiniteVolume_Parm.ID_Lambda = 0;
                {
                    std::vector<double> Ub(U, U + tot), L(tot);
                    fill_ghosts(c, Ub.data());
                    compute_dudt(c, parm, Ub.data(), L.data(), &cmax);
                }
                double dt_re = est_dt(c, cmax);
                if (time == 0.0) dt_prev = dt_re;
                if (c->change_limiter && dt_prev > 0.0) dt_re = std::min(dt_re, 1.1 * dt_prev);
                dt0 = dt_re;
                const double eps2 = 1.0e-3 * dt0;
                if (time + dt0 > stop_time - eps2) dt0 = stop_time - time;
                dt_prev = dt0;
                const int again = rk3_step(c, parm, U, dt0, &cmax);
                parm.FiniteVolume_Parm.ID_Lambda = 1;
                if (again) {
                    // this engine's convention: the state the step started from is kept and the run stops
                    std::memcpy(U, Usave.data(), sizeof(double) * tot);
                    throw std::runtime_error("the energy bound failed again after the step was taken again");
                }
            }
            if (dts) dts[step] = dt0;
            time += dt0;
            ++taken;
        }
        *t = time;
    });
    return rc == 0 ? taken : rc;
}

int cmp_pf_step(const cmp_case* c, const cmp_pf* pf, double* U, double dt, double* info) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    return guarded([&] { pf_step(c, pf, U, dt, info); });
#else
    (void)c; (void)pf; (void)U; (void)dt; (void)info;
    return -2;
#endif
}

int cmp_pf_grad_q(const cmp_case* c, const cmp_pf* pf, const double* U, double dt, double* gq0, double* gq1,
                  double* gq2, double* info) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    return guarded([&] {
        PfSetup S = pf_setup(c, pf, U);
        std::vector<FField> GQ;
        pf_grad_q(c, pf, S, U, dt, GQ, info);
        double* out[3] = {gq0, gq1, gq2};
        for (int d = 0; d < AMREX_SPACEDIM; ++d)
            if (out[d]) std::memcpy(out[d], GQ[d].v.data(), GQ[d].v.size() * sizeof(double));
    });
#else
    (void)c; (void)pf; (void)U; (void)dt; (void)gq0; (void)gq1; (void)gq2; (void)info;
    return -2;
#endif
}

int cmp_pf_dudt(const cmp_case* c, const cmp_pf* pf, const double* U, const double* gq0, const double* gq1,
                const double* gq2, double* dUdt) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    return guarded([&] {
        PfSetup S = pf_setup(c, pf, U);
        Parm parm = make_parm(c);
        parm.PhaseField_Parm = S.P;
        Geo g(c);
        const double* in[3] = {gq0, gq1, gq2};
        std::vector<FField> GQ(AMREX_SPACEDIM);
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
            GQ[d] = FField(g, d);
            std::memcpy(GQ[d].v.data(), in[d], GQ[d].v.size() * sizeof(double));
        }
        std::vector<double> Ub(U, U + g.S * NSTATE);
        fill_ghosts(c, Ub.data());
        pf_compute_dudt(c, parm, Ub.data(), GQ, dUdt);
    });
#else
    (void)c; (void)pf; (void)U; (void)gq0; (void)gq1; (void)gq2; (void)dUdt;
    return -2;
#endif
}

int cmp_advance_pf(const cmp_case* c, const cmp_pf* pf, double* U, int nsteps, double stop_time, double* t,
                   double* dts) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    int taken = 0;
    int rc = guarded([&] {
        Parm parm = make_parm(c);
        Geo g(c);
        double dt_prev = 1.e100;
        double cmax = 0.0;
        double time = *t;
        for (int step = 0; step < nsteps && time < stop_time; ++step) {
            if (time == 0.0) {
                std::vector<double> Ub(U, U + g.S * NSTATE), L(g.S * NSTATE);
                fill_ghosts(c, Ub.data());
                compute_dudt(c, parm, Ub.data(), L.data(), &cmax);
            }
            double dt_est = est_dt(c, cmax);
            if (time == 0.0) dt_prev = dt_est;
            if (c->change_limiter && dt_prev > 0.0) dt_est = std::min(dt_est, 1.1 * dt_prev);
            double dt0 = dt_est;
            const double eps = 1.0e-3 * dt0;
            if (time + dt0 > stop_time - eps) dt0 = stop_time - time;
            dt_prev = dt0;
            rk3_step(c, parm, U, dt0, &cmax);
            pf_step(c, pf, U, dt0, nullptr);
            if (dts) dts[step] = dt0;
            time += dt0;
            ++taken;
        }
        *t = time;
    });
    return rc == 0 ? taken : rc;
#else
    (void)c; (void)pf; (void)U; (void)nsteps; (void)stop_time; (void)t; (void)dts;
    return -2;
#endif
}

int cmp_amr_advance(const cmp_case* c, int nlev, const cmp_amr_box* boxes, int nbox, double** U, int nsteps,
                    double stop_time, double* t, double* dts) {
    int taken = 0;
    int rc = guarded([&] { taken = amr_advance(c, nlev, boxes, nbox, U, nsteps, stop_time, t, dts); });
    return rc == 0 ? taken : rc;
}

// ErrorEst of one level (source/COMPAS.cpp:767-932) for the tagging criteria of that level, with the
// reference's own Tagging.H tests and compute_derived_var; the Derived scratch array covers the
// valid cells grown by one (ngrow = 1), as ErrorEst's.
int cmp_tag(const cmp_case* c, const double* cv, const double* U, const cmp_tag_crit* crit, int ncrit,
            unsigned char* tags) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    try {
        Geo g(c);
        Parm parm = make_parm(c);
        parm.cv_1 = cv[0];
        parm.cv_2 = cv[1];
        auto st = g.view(const_cast<double*>(U), NSTATE);
        amrex::Array4<amrex::Real const> stc(st);
        std::vector<double> der((size_t)g.S, 0.0);
        auto dv = g.view(der.data(), 1);
        std::vector<char> tg((size_t)g.nx * g.ny * g.nz, 0);
        amrex::Array4<char> tagfab(tg.data(), amrex::Dim3{0, 0, 0}, amrex::Dim3{g.nx, g.ny, g.nz}, 1);
        const double dx = c->dx[0], dy = c->dx[1], dz = (AMREX_SPACEDIM == 3) ? c->dx[2] : 1.0;
        const char tagval = 1;
        const int gz1 = (AMREX_SPACEDIM == 3) ? 1 : 0;
        for (int v = 0; v < ncrit; ++v) {
            const cmp_tag_crit& cr = crit[v];
            amrex::Array4<amrex::Real> varfab = st;
            int comp = cr.var;
            if (cr.derived) {
                for (int k = -gz1; k < g.nz + gz1; ++k)
                for (int j = -1; j < g.ny + 1; ++j)
                for (int i = -1; i < g.nx + 1; ++i)
                    compute_derived_var(i, j, k, cr.var, dx, dy, dz, dv, stc, parm);
                varfab = dv;
                comp = 0;
            }
            for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                if (cr.kind == 0) state_grad(i, j, k, comp, tagfab, varfab, cr.v0, tagval);
                else if (cr.kind == 1) state_value_less(i, j, k, comp, tagfab, varfab, cr.v0, tagval);
                else if (cr.kind == 2) state_value_greater(i, j, k, comp, tagfab, varfab, cr.v0, tagval);
                else state_value_range(i, j, k, comp, tagfab, varfab, cr.v0, cr.v1, tagval);
            }
        }
        for (size_t q = 0; q < tg.size(); ++q) tags[q] = (unsigned char)tg[q];
        return 0;
    } catch (...) {
        return -1;
    }
#else
    (void)c; (void)cv; (void)U; (void)crit; (void)ncrit; (void)tags;
    return -2;
#endif
}

// Plot variables (PlotFileMF with compute_derived_var, source/COMPAS.cpp:2483-2511) of the valid cells.
int cmp_derive(const cmp_case* c, const double* cv, const double* U, const int* vars, const int* derived, int nvars,
               double* out) {
#if (PHYSICS == FIVEEQS || PHYSICS == SIXEQS)
    try {
        Geo g(c);
        Parm parm = make_parm(c);
        parm.cv_1 = cv[0];
        parm.cv_2 = cv[1];
        auto st = g.view(const_cast<double*>(U), NSTATE);
        amrex::Array4<amrex::Real const> stc(st);
        std::vector<double> one((size_t)g.S, 0.0);
        auto ov = g.view(one.data(), 1);
        const double dx = c->dx[0], dy = c->dx[1], dz = (AMREX_SPACEDIM == 3) ? c->dx[2] : 1.0;
        const long long cells = (long long)g.nx * g.ny * g.nz;
        for (int v = 0; v < nvars; ++v)
            for (int k = 0; k < g.nz; ++k)
                for (int j = 0; j < g.ny; ++j)
                    for (int i = 0; i < g.nx; ++i) {
                        const long long t = ((long long)k * g.ny + j) * g.nx + i;
                        double val;
                        if (derived[v]) {
                            compute_derived_var(i, j, k, vars[v], dx, dy, dz, ov, stc, parm);
                            val = ov(i, j, k, 0);
                        } else {
                            val = st(i, j, k, vars[v]);
                        }
                        out[v * cells + t] = val;
                    }
        return 0;
    } catch (...) {
        return -1;
    }
#else
    (void)c; (void)cv; (void)U; (void)vars; (void)derived; (void)nvars; (void)out;
    return -2;
#endif
}

int cmp_thinc_face(const double* beta, const double* sigma, const double* abar, const int* side, long long n,
                   double* out) {
    for (long long t = 0; t < n; ++t) out[t] = Reconstruction2Face_THINC_D(beta[t], sigma[t], abar[t], side[t]);
    return 0;
}

}  // extern "C"
