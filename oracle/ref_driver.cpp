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

#include <Physics_Compressible_TwoPhase.H>
#if (PHYSICS == FIVEEQS)
#include <Physics_Compressible5Eq.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
#include <Operators_Compressible5Eq.H>
#elif (PHYSICS == SIXEQS)
#include <RelaxationPressure_Safeguarded.H>
#include <Physics_Compressible6Eq.H>
#include <Operators_FV.H>
#include <Operators_FD.H>
#include <Operators_Compressible6Eq.H>
#endif

#include "oracle_api.h"

#include <cstring>
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
    p.A1 = c->A1; p.A2 = c->A2; p.B1 = c->B1; p.B2 = c->B2;
    p.C1 = c->C1; p.C2 = c->C2; p.D1 = c->D1; p.D2 = c->D2;
    auto& fv = p.FiniteVolume_Parm;
    fv.ID_WENO = 1;
    fv.ID_Limiter = c->id_limiter;
    fv.ID_Poly = 4;
    fv.Num_Grow = 3;
    fv.Scheme = (c->id_limiter == 6) ? FVReconstruction::WENO_5B : FVReconstruction::WENO_5;
    fv.Quadrature_Weight = 1.0 / 12.0;
    fv.ID_THINC = c->thinc;
    fv.ID_THINC_UseNormal = c->thinc_use_normal;
    fv.THINC_EPS = c->thinc_eps;
    fv.THINC_Beta = c->thinc_beta;
    fv.THINC_NormalThreshold = c->thinc_normal_threshold;
    p.Physics_Parm.ID_Riemann = c->id_riemann;
#if (PHYSICS == FIVEEQS)
    p.Physics_Parm.source_term = c->source_term;
#elif (PHYSICS == SIXEQS)
    p.Physics_Parm.pressure_relaxation = c->relaxation;
    p.Physics_Parm.pressure_relaxation_trace = c->relax_trace;
    p.Physics_Parm.relaxation = c->relaxation;
#endif
    return p;
}

// AMReX BCType for component n in direction d at code `code`
// (source/Class_Compressible6Eq_PhaseField.cpp:362-431): 0 int_dir, 2 foextrap, 3/4 reflect_even
// (normal momentum reflect_odd), 5 reflect_odd for every momentum component.
enum { BC_INT = 0, BC_FOEXTRAP = 1, BC_EVEN = 2, BC_ODD = 3 };
int bc_kind(int code, int n, int d) {
    const bool mom = (n >= 2 && n < 2 + AMREX_SPACEDIM);
    const bool normal = mom && (n - 2 == d);
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
void compute_dudt(const cmp_case* c, const Parm& parm, const double* U, double* dUdt, double* cmax_out) {
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
}

void relax(const cmp_case* c, const Parm& parm, double* U) {
#if (PHYSICS == SIXEQS)
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

// ThirdOrderSSPRK: the stage combinations as MultiFab::LinComb / Saxpy compute them
// (dst = a*x + b*y, then dst += a*x), with PostTimeStage (relaxation) after each stage.
void rk3_step(const cmp_case* c, const Parm& parm, double* U, double dt, double* cmax_out) {
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
    if (cmax_out) *cmax_out = cm;
}

double est_dt(const cmp_case* c, double cmax) {
    double dt = std::numeric_limits<double>::max();
    for (int d = 0; d < AMREX_SPACEDIM; ++d) dt = amrex::min(dt, c->cfl * c->dx[d] / cmax);
    return dt;
}

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
    return guarded([&] {
        Parm parm = make_parm(c);
        rk3_step(c, parm, U, dt, cmax);
    });
}

int cmp_advance(const cmp_case* c, double* U, int nsteps, double stop_time, double* t, double* dts) {
    int taken = 0;
    int rc = guarded([&] {
        Parm parm = make_parm(c);
        Geo g(c);
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
            rk3_step(c, parm, U, dt0, &cmax);
            if (dts) dts[step] = dt0;
            time += dt0;
            ++taken;
        }
        *t = time;
    });
    return rc == 0 ? taken : rc;
}

}  // extern "C"
