// C-ABI of the B200 right-hand-side engine: parameters (the reference's inputs keys), the drop-in
// stage kernels on caller-owned device arrays, and a single-level advance whose time-step control
// runs on the device (no host synchronisation inside a run, CUDA-graph replay per step).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <map>
#include <mutex>
#include <vector>

#include "compas_b200.h"
#include "physics.cuh"
#include "relax.cuh"
#include "launch.h"
#include "phasefield.h"
#include "stage_kernel.cuh"
#include "bound.cuh"

namespace compas {

// ------------------------------------------------------------------------------------------------
// error reporting
// ------------------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(COMPAS_B200_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------------------------------------
// small kernels: boundary fill, stand-alone relaxation, step control
// ------------------------------------------------------------------------------------------------

// AMReX BCType of component n across a face normal to d for a COMPAS boundary code
// (source/Class_Compressible6Eq_PhaseField.cpp:352-434, Class_Compressible5Eq_PhaseField.cpp:162-):
// 0 int_dir (periodic), 2 foextrap, 3/4 reflect_even with the normal momentum reflect_odd,
// 5 reflect_odd for every momentum component. The momentum components are m0 .. m0 + D - 1 (m0 = 2
// for the two-phase models, NPHASE for FIVEEQS_NPHASE,
// source/Class_Compressible5Eq_NPhase_PhaseField.cpp:133-205).
enum { kBcPeriodic = 0, kBcExtrap = 1, kBcEven = 2, kBcOdd = 3 };

__device__ __forceinline__ int bc_kind(int code, int n, int d, int D, int m0) {
    const bool mom = (n >= m0 && n < m0 + D);
    switch (code) {
        case 0: return kBcPeriodic;
        case 2: return kBcExtrap;
        case 3:
        case 4: return (mom && n - m0 == d) ? kBcOdd : kBcEven;
        default: return mom ? kBcOdd : kBcEven;  // 5: no-slip wall
    }
}

struct BcArgs {
    double* U;
    Grid g;
    int N, D, m0;
    int lo[3], hi[3];
};

// Map one coordinate of a ghost cell to its source along d; returns the sign factor.
__device__ __forceinline__ double bc_map(int& x, int len, int code_lo, int code_hi, int n, int d, int D, int m0) {
    if (x < 0) {
        const int kind = bc_kind(code_lo, n, d, D, m0);
        if (kind == kBcPeriodic) { x += len; return 1.0; }
        if (kind == kBcExtrap) { x = 0; return 1.0; }
        x = -1 - x;
        return kind == kBcOdd ? -1.0 : 1.0;
    }
    if (x >= len) {
        const int kind = bc_kind(code_hi, n, d, D, m0);
        if (kind == kBcPeriodic) { x -= len; return 1.0; }
        if (kind == kBcExtrap) { x = len - 1; return 1.0; }
        x = 2 * len - 1 - x;
        return kind == kBcOdd ? -1.0 : 1.0;
    }
    return 1.0;
}

// One thread per ghost cell (all components). Ghost cells are enumerated as the z slabs (full
// padded planes), then the y slabs of the valid z range, then the x slabs of the valid y, z range.
// Filling x, then y, then z over the full extent of the other directions (the oracle's order)
// gives at every ghost cell the valid cell found by mapping each coordinate independently, with
// the product of the per-direction signs, which is what this kernel computes directly.
__host__ __device__ __forceinline__ long long ghost_count(const Grid& g) {
    return 2LL * g.gz * g.pxy + 2LL * g.ng * g.px * g.n[2] + 2LL * g.ng * g.n[1] * g.n[2];
}

// Ghost cell (i, j, k) of U from the valid cell its coordinates map to, all components.
__device__ __forceinline__ void fill_cell(double* U, const Grid& g, int N, int D, int m0, const int* lo,
                                          const int* hi, int i, int j, int k) {
    const long long dst = g.at(i, j, k);
    for (int n = 0; n < N; ++n) {
        int si = i, sj = j, sk = k;
        double sgn = bc_map(si, g.n[0], lo[0], hi[0], n, 0, D, m0);
        sgn *= bc_map(sj, g.n[1], lo[1], hi[1], n, 1, D, m0);
        if (D == 3) sgn *= bc_map(sk, g.n[2], lo[2], hi[2], n, 2, D, m0);
        U[n * g.S + dst] = sgn * U[n * g.S + g.at(si, sj, sk)];
    }
}

// Fill ghost cell number q (enumeration above) of U, all components.
__device__ __forceinline__ void fill_ghost_cell(double* U, const Grid& g, int N, int D, int m0, const int* lo,
                                                const int* hi, long long q) {
    const long long PX = g.px, PY = g.pxy / g.px;
    const long long nz_slab = 2LL * g.gz * PX * PY;
    const long long ny_slab = 2LL * g.ng * PX * g.n[2];
    {
        int i, j, k;
        if (q < nz_slab) {
            const long long plane = PX * PY;
            const int s = (int)(q / plane);
            const long long r = q % plane;
            i = (int)(r % PX) - g.ng;
            j = (int)(r / PX) - g.ng;
            k = (s < g.gz) ? s - g.gz : g.n[2] + (s - g.gz);
        } else if (q < nz_slab + ny_slab) {
            const long long r0 = q - nz_slab;
            const long long row = PX * g.n[2];
            const int s = (int)(r0 / row);
            const long long r = r0 % row;
            i = (int)(r % PX) - g.ng;
            k = (int)(r / PX);
            j = (s < g.ng) ? s - g.ng : g.n[1] + (s - g.ng);
        } else {
            const long long r0 = q - nz_slab - ny_slab;
            const long long col = (long long)g.n[1] * g.n[2];
            const int s = (int)(r0 / col);
            const long long r = r0 % col;
            j = (int)(r % g.n[1]);
            k = (int)(r / g.n[1]);
            i = (s < g.ng) ? s - g.ng : g.n[0] + (s - g.ng);
        }
        fill_cell(U, g, N, D, m0, lo, hi, i, j, k);
    }
}

__global__ void fill_boundary_kernel(BcArgs a) {
    const long long total = ghost_count(a.g);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x)
        fill_ghost_cell(a.U, a.g, a.N, a.D, a.m0, a.lo, a.hi, q);
}

// The ghost cells of a slab of the padded box: the padded planes (3D: z planes; 2D: y rows) l0 <= l < l1
// of the slowest direction, in valid coordinates (ghost planes negative or >= n). Every ghost cell
// maps to the valid cell fill_boundary_kernel maps it to; the slab's own planes hold every source
// unless the slab direction is periodic.
__global__ void fill_boundary_slab_kernel(BcArgs a, int l0, int l1) {
    const Grid& g = a.g;
    const long long PX = g.px, PY = g.pxy / g.px;
    const long long unit = (a.D == 3) ? PX * PY : PX;
    const long long total = (long long)(l1 - l0) * unit;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int l = l0 + (int)(q / unit);
        const long long r = q % unit;
        const int i = (int)(r % PX) - g.ng;
        int j, k;
        if (a.D == 3) {
            j = (int)(r / PX) - g.ng;
            k = l;
        } else {
            j = l;
            k = 0;
        }
        const bool valid = i >= 0 && i < g.n[0] && j >= 0 && j < g.n[1] && k >= 0 && k < g.n[2];
        if (!valid) fill_cell(a.U, g, a.N, a.D, a.m0, a.lo, a.hi, i, j, k);
    }
}

template <int D>
__global__ void relax_kernel(double* U, Grid g, Eos e, double trace, unsigned int* err) {
    constexpr int N = SixEq<D>::N;
    const long long cells = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.n[0]);
        const int j = (int)((c / g.n[0]) % g.n[1]);
        const int k = (int)(c / ((long long)g.n[0] * g.n[1]));
        const long long q = g.at(i, j, k);
        double v[N];
        for (int n = 0; n < N; ++n) v[n] = U[n * g.S + q];
        relax_pressure<D>(v, e, trace, err);
        for (int n = 0; n < N; ++n) U[n * g.S + q] = v[n];
    }
}

// Device-resident time-step control of one level (COMPAS::ComputeDt, source/COMPAS.cpp:2249-2303,
// and the coarse-step loop of Compressible_PhaseField::Evolve, source/Class_Compressible_PhaseField.cpp:201).
struct StepCtl {
    double t;
    double dt;
    double dt_prev;             // COMPAS dt[lev], 1e100 before the first step (source/COMPAS.cpp:81)
    double stop_time;
    unsigned long long cmax;    // bits of the largest face speed of the last step's stages
    int steps;
    int done;
    unsigned int err;
    int pad;
};

struct StepParams {
    double cfl;
    double dx[3];
    int D;
    int limiter;
    double* dts;
    int dts_cap;
};

__global__ void step_begin_kernel(StepCtl* s, StepParams p) {
    if (s->done) return;
    if (!(s->t < s->stop_time)) {
        s->done = 1;
        return;
    }
    const double cmax = __longlong_as_double((long long)s->cmax);
    double dt_est = DBL_MAX;
    for (int d = 0; d < p.D; ++d) dt_est = dmin(dt_est, p.cfl * p.dx[d] / cmax);
    if (s->t == 0.0) s->dt_prev = dt_est;
    if (p.limiter && s->dt_prev > 0.0) dt_est = dmin(dt_est, 1.1 * s->dt_prev);
    double dt0 = dt_est;
    const double eps = 1.0e-3 * dt0;
    if (s->t + dt0 > s->stop_time - eps) dt0 = s->stop_time - s->t;
    if (!(dt0 > 0.0) || !(dt0 <= DBL_MAX)) {
        s->err |= COMPAS_B200_ERR_CFL;
        s->done = 1;
        return;
    }
    s->dt = dt0;
    s->dt_prev = dt0;
    s->cmax = 0ull;  // stage 0 resets c_max (source/Class_Compressible_PhaseField.cpp:3162-3164)
    if (p.dts && s->steps < p.dts_cap) p.dts[s->steps] = dt0;
}

__global__ void step_end_kernel(StepCtl* s) {
    if (s->done) return;
    s->t += s->dt;
    s->steps += 1;
}

__global__ void set_time_kernel(StepCtl* s, double t0, double stop_time, int reset) {
    if (reset) {
        s->t = t0;
        s->dt = 0.0;
        s->dt_prev = 1.e100;
        s->cmax = 0ull;
        s->steps = 0;
        s->err = 0u;
    }
    s->stop_time = stop_time;
    s->done = 0;
}

// ------------------------------------------------------------------------------------------------
// launch helpers
// ------------------------------------------------------------------------------------------------
static Grid make_grid(const compas_b200_parm* p, const compas_b200_geom* g) {
    Grid G;
    G.n[0] = g->n[0];
    G.n[1] = g->n[1];
    G.n[2] = (p->dim == 3) ? g->n[2] : 1;
    G.ng = g->ng;
    G.gz = (p->dim == 3) ? g->ng : 0;
    G.px = G.n[0] + 2 * G.ng;
    const long long py = G.n[1] + 2 * G.ng;
    const long long pz = G.n[2] + 2 * G.gz;
    G.pxy = G.px * py;
    G.S = G.pxy * pz;
    G.dx[0] = g->dx[0];
    G.dx[1] = g->dx[1];
    G.dx[2] = (p->dim == 3) ? g->dx[2] : 1.0;
    return G;
}

static Eos make_eos(const compas_b200_parm* p) {
    Eos e;
    std::memset(&e, 0, sizeof(e));
    e.A1 = p->A1; e.A2 = p->A2; e.B1 = p->B1; e.B2 = p->B2;
    e.C1 = p->C1; e.C2 = p->C2; e.D1 = p->D1; e.D2 = p->D2;
    e.iA1 = 1.0 / p->A1;
    e.iA2 = 1.0 / p->A2;
    e.pinf1 = p->B1 / (p->A1 + 1.0);
    e.pinf2 = p->B2 / (p->A2 + 1.0);
    if (p->source_term == 1) {
        e.pmin1 = -p->B1 / (p->A1 + 1.0);
        e.pmin2 = -p->B2 / (p->A2 + 1.0);
    } else {
        e.pmin1 = -p->B1 / p->A1;
        e.pmin2 = -p->B2 / p->A2;
    }
    for (int k = 0; k < kMaxPhases; ++k) {
        e.Ak[k] = p->Ak[k];
        e.Bk[k] = p->Bk[k];
        e.Ck[k] = p->Ck[k];
        e.Dk[k] = p->Dk[k];
        e.pmink[k] = (p->source_term == 1) ? -p->Bk[k] / (p->Ak[k] + 1.0) : -p->Bk[k] / p->Ak[k];
    }
    e.fA1 = (float)p->A1; e.fA2 = (float)p->A2;
    e.fB1 = (float)p->B1; e.fB2 = (float)p->B2;
    e.fC1 = (float)p->C1; e.fC2 = (float)p->C2;
    return e;
}

// NSTATE (include/Macros.H:73, :89, :114).
static int nstate_of(int physics, int dim, int nphase) {
    if (physics == COMPAS_B200_FIVEEQS_NPHASE) return 2 * nphase + dim + 1;
    if (physics == COMPAS_B200_SIXEQS_IE_NPHASE) return 3 * nphase + dim + 1;
    return (physics == COMPAS_B200_FIVEEQS ? 4 : 5) + dim;
}
static int nstate(const compas_b200_parm* p) { return nstate_of(p->physics, p->dim, p->nphase); }

// First momentum component (INDEX_MomentumX).
static int mom0_of(int physics, int nphase) {
    return physics == COMPAS_B200_FIVEEQS_NPHASE ? nphase : (physics == COMPAS_B200_SIXEQS_IE_NPHASE ? 3 * nphase : 2);
}

// The models with per-phase EOS lists (prob.EOS.gamma, ... with NPHASE values each).
static bool nphase_model(int physics) {
    return physics == COMPAS_B200_FIVEEQS_NPHASE || physics == COMPAS_B200_SIXEQS_IE_NPHASE;
}

// The N-phase kernels this build instantiates.
static bool nphase_built(int dim, int nphase) {
    return (dim == 2 && nphase >= 2 && nphase <= 4) || (dim == 3 && nphase == 3);
}
static bool sixn_built(int dim, int nphase) { return (dim == 2 && (nphase == 2 || nphase == 3)) || (dim == 3 && nphase == 3); }

static int check_args(const compas_b200_parm* p, const compas_b200_geom* g) {
    if (!p || !g) return fail(COMPAS_B200_EARG, "null parameter or geometry");
    if (p->physics != COMPAS_B200_FIVEEQS && p->physics != COMPAS_B200_SIXEQS &&
        p->physics != COMPAS_B200_FIVEEQS_NPHASE && p->physics != COMPAS_B200_SIXEQS_IE_NPHASE)
        return fail(COMPAS_B200_EARG, "physics must be FIVEEQS (555), SIXEQS (666), FIVEEQS_NPHASE (55501) or "
                                      "SIXEQS_IE_NPHASE (66601)");
    if (p->dim != 2 && p->dim != 3) return fail(COMPAS_B200_EARG, "dim must be 2 or 3");
    if (p->physics == COMPAS_B200_FIVEEQS_NPHASE) {
        if (!nphase_built(p->dim, p->nphase))
            return fail(COMPAS_B200_EUNSUPPORTED, "FIVEEQS_NPHASE: this build runs NPHASE 2, 3, 4 in 2D and 3 in 3D");
        if (p->thinc) return fail(COMPAS_B200_EUNSUPPORTED, "FIVEEQS_NPHASE: FiniteVolume.THINC is not in this engine");
    }
    if (p->physics == COMPAS_B200_SIXEQS_IE_NPHASE) {
        if (!sixn_built(p->dim, p->nphase))
            return fail(COMPAS_B200_EUNSUPPORTED, "SIXEQS_IE_NPHASE: this build runs NPHASE 2, 3 in 2D and 3 in 3D");
        if (p->thinc) return fail(COMPAS_B200_EUNSUPPORTED, "SIXEQS_IE_NPHASE: FiniteVolume.THINC is not in this engine");
        if (p->phase_field)
            return fail(COMPAS_B200_EUNSUPPORTED, "PhaseField.phase_field = 1: this engine runs the FIVEEQS and SIXEQS "
                                                  "Phase-Field step");
        if (p->id_bound)
            return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1: the bound-preserving right-hand side is "
                                                  "the five-equation models' (FIVEEQS, FIVEEQS_NPHASE)");
    }
    if (p->id_weno ? (p->id_limiter < 3 || p->id_limiter > 6)
                   : (p->id_limiter < 0 || p->id_limiter > 4))
        return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.Scheme: this build runs GODUNOV, MUSCL-*, WENO3, WENO3B, "
                                              "WENO5 and WENO5B");
    if (p->id_limiter < 5 && !p->id_bound && (p->thinc || p->phase_field))
        return fail(COMPAS_B200_EUNSUPPORTED, "THINC and the Phase-Field step run with WENO5 / WENO5B here");
    if (p->id_riemann < 0 || p->id_riemann > 2)
        return fail(COMPAS_B200_EUNSUPPORTED, "Physics.RiemannSolver: this build runs LLF, HLL and HLLC");
    if (p->phase_field && p->physics == COMPAS_B200_FIVEEQS_NPHASE)
        return fail(COMPAS_B200_EUNSUPPORTED, "PhaseField.phase_field = 1: this engine runs the FIVEEQS and SIXEQS "
                                              "Phase-Field step");
    if (p->phase_field && p->pf_mechanism != 1 && p->pf_mechanism != 3)
        return fail(COMPAS_B200_EUNSUPPORTED, "PhaseField.Mechanism: this engine runs CAC-Adv and ACDI");
    if (p->phase_field && p->pf_explicit_rc && p->pf_mechanism == 1)
        return fail(COMPAS_B200_EARG, "non flux-based mechanism can not use the explicit RC approach");
    if (p->precision != 0 && p->precision != 1)
        return fail(COMPAS_B200_EARG, "precision must be 0 (plain FP64) or 1 (mixed)");
    if (p->id_bound) {
        // the bound-preserving branch of the flux functor is the five-equation model's
        // (include/Operators_Compressible5Eq/FVM_Conservative2FluxHyperbolic_K_Compressible5Eq.H:100-152)
        if (p->physics == COMPAS_B200_SIXEQS)
            return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1: the bound-preserving right-hand side is "
                                                  "the five-equation models' (FIVEEQS, FIVEEQS_NPHASE)");
        if (p->precision != 0)
            return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1 runs in plain FP64 (compas_b200.precision = fp64)");
        if (p->phase_field)
            return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1 with PhaseField.phase_field = 1 is not in "
                                                  "this engine");
        if (p->id_lambda != 0 && p->id_lambda != 1) return fail(COMPAS_B200_EARG, "id_lambda must be 0 or 1");
    }
    if (g->ng < 3) return fail(COMPAS_B200_EARG, "WENO5 needs ng >= 3 ghost cells");
    for (int d = 0; d < p->dim; ++d) {
        if (g->n[d] < 1) return fail(COMPAS_B200_EARG, "empty box");
        if (!(g->dx[d] > 0.0)) return fail(COMPAS_B200_EARG, "cell sizes must be positive");
        for (int code : {g->lo_bc[d], g->hi_bc[d]})
            if (code != 0 && code != 2 && code != 3 && code != 4 && code != 5)
                return fail(COMPAS_B200_EARG, "boundary codes: 0 interior, 2 outflow, 3 symmetry, 4 slip wall, "
                                              "5 no-slip wall (1 inflow needs a user function)");
        if ((g->lo_bc[d] == 0) != (g->hi_bc[d] == 0))
            return fail(COMPAS_B200_EARG, "a periodic direction needs code 0 on both sides");
        if (g->lo_bc[d] == 0 && g->n[d] < g->ng)
            return fail(COMPAS_B200_EARG, "a periodic direction needs at least ng cells");
        for (int code : {g->lo_bc[d], g->hi_bc[d]})
            if (code != 0 && code != 2 && g->n[d] < g->ng)
                return fail(COMPAS_B200_EARG, "a reflecting boundary needs at least ng cells");
    }
    if (p->dim == 2 && g->n[2] != 1) return fail(COMPAS_B200_EARG, "n[2] must be 1 in 2D");
    return COMPAS_B200_OK;
}

// The stage kernel of the model, dimension and scheme of p (kernels live in kern_*.cu).
static KernelChoice choice_of(const compas_b200_parm* p) {
    KernelChoice k;
    k.limiter = p->id_limiter;
    k.precision = p->precision;
    k.thinc = p->thinc;
    k.phase_field = 0;
    k.shape = 0;
    return k;
}

static int launch_stage(const compas_b200_parm* p, const StageArgs& a, cudaStream_t st, int phase_field = 0,
                        int shape = 0, const TmaMaps* tm = nullptr) {
    const int ts = (p->dim == 2) ? kTile2 : kTile3;
    const long long tiles = (long long)((a.g.n[0] + ts - 1) / ts) * ((a.g.n[1] + ts - 1) / ts) *
                            ((a.g.n[2] + (p->dim == 2 ? 1 : ts) - 1) / (p->dim == 2 ? 1 : ts));
    if (tiles > 0x7fffffffLL) return fail(COMPAS_B200_EARG, "box too large");
    KernelChoice k = choice_of(p);
    k.shape = shape;
    if (phase_field) {
        k.thinc = 0;
        k.phase_field = 1;
    }
    cudaError_t e;
    if (p->physics == COMPAS_B200_FIVEEQS)
        e = (p->dim == 2) ? launch_stage_fiveeq2(k, a, st, tm) : launch_stage_fiveeq3(k, a, st, tm);
    else if (p->physics == COMPAS_B200_SIXEQS)
        e = (p->dim == 2) ? launch_stage_sixeq2(k, a, st, tm) : launch_stage_sixeq3(k, a, st, tm);
    else if (p->physics == COMPAS_B200_SIXEQS_IE_NPHASE)
        e = (p->dim == 3) ? launch_stage_sixeqn3_3(k, a, st, tm)
            : (p->nphase == 2) ? launch_stage_sixeqn2_2(k, a, st, tm) : launch_stage_sixeqn2_3(k, a, st, tm);
    else if (p->dim == 3) e = launch_stage_fiveeqn3_3(k, a, st, tm);
    else e = (p->nphase == 2) ? launch_stage_fiveeqn2_2(k, a, st, tm)
           : (p->nphase == 3) ? launch_stage_fiveeqn2_3(k, a, st, tm) : launch_stage_fiveeqn2_4(k, a, st, tm);
    if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("stage kernel launch: ") + cudaGetErrorString(e));
    return COMPAS_B200_OK;
}

static int launch_list(int physics, int dim, int nphase, int limiter, int precision, const ListArgs& L,
                       cudaStream_t st, int shape = 0) {
    KernelChoice k;
    k.limiter = limiter;
    k.precision = precision;
    k.thinc = 0;
    k.phase_field = 0;
    k.shape = shape;
    cudaError_t e;
    if (physics == COMPAS_B200_FIVEEQS) e = (dim == 2) ? launch_list_fiveeq2(k, L, st) : launch_list_fiveeq3(k, L, st);
    else if (physics == COMPAS_B200_SIXEQS) e = (dim == 2) ? launch_list_sixeq2(k, L, st) : launch_list_sixeq3(k, L, st);
    else if (physics == COMPAS_B200_SIXEQS_IE_NPHASE)
        e = (dim == 3) ? launch_list_sixeqn3_3(k, L, st)
            : (nphase == 2) ? launch_list_sixeqn2_2(k, L, st) : launch_list_sixeqn2_3(k, L, st);
    else if (dim == 3) e = launch_list_fiveeqn3_3(k, L, st);
    else e = (nphase == 2) ? launch_list_fiveeqn2_2(k, L, st)
           : (nphase == 3) ? launch_list_fiveeqn2_3(k, L, st) : launch_list_fiveeqn2_4(k, L, st);
    if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("box-list kernel launch: ") + cudaGetErrorString(e));
    return COMPAS_B200_OK;
}

static int launch_fill(const compas_b200_parm* p, const compas_b200_geom* geo, double* U, cudaStream_t st) {
    BcArgs b;
    b.U = U;
    b.g = make_grid(p, geo);
    b.N = nstate(p);
    b.D = p->dim;
    b.m0 = mom0_of(p->physics, p->nphase);
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = geo->lo_bc[d];
        b.hi[d] = geo->hi_bc[d];
    }
    const Grid& g = b.g;
    const long long total = 2LL * g.gz * g.pxy + 2LL * g.ng * g.px * g.n[2] + 2LL * g.ng * g.n[1] * g.n[2];
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148LL * 16) blocks = 148LL * 16;
    if (blocks < 1) blocks = 1;
    fill_boundary_kernel<<<(unsigned)blocks, threads, 0, st>>>(b);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

// The ghost cells of the slab l0 <= l < l1 (fill_boundary_slab_kernel).
static int launch_fill_slab(const compas_b200_parm* p, const compas_b200_geom* geo, double* U, int l0, int l1,
                            cudaStream_t st) {
    BcArgs b;
    b.U = U;
    b.g = make_grid(p, geo);
    b.N = nstate(p);
    b.D = p->dim;
    b.m0 = mom0_of(p->physics, p->nphase);
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = geo->lo_bc[d];
        b.hi[d] = geo->hi_bc[d];
    }
    const long long unit = (p->dim == 3) ? b.g.pxy : b.g.px;
    const long long total = (long long)(l1 - l0) * unit;
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148LL * 16) blocks = 148LL * 16;
    if (blocks < 1) blocks = 1;
    fill_boundary_slab_kernel<<<(unsigned)blocks, threads, 0, st>>>(b, l0, l1);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

// ------------------------------------------------------------------------------------------------
// Autotuner: the launch shape (threads per CTA, CTAs per SM; kern_impl.cuh) and the tile traversal
// order (tile_coords) of the plain stage kernels, picked per model, precision and box size by timing
// every candidate on the caller's own data (one RK stage each, CUDA events, after one warm-up
// launch) the first time a level or batch advances. Every candidate computes the same faces with
// the same arithmetic, so the choice changes the time, never the result. Choices are cached for the
// process, keyed by model, scheme, precision, kind (single box / box list) and size.
// ------------------------------------------------------------------------------------------------
struct TuneChoice {
    int shape = 0, order = 0;
    int tma = 0;  // halo slabs staged by TMA (single-box 3D mixed kernels that have tensor maps)
    float ms = 0.f;
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneChoice> g_tune_cache;

static std::string tune_key(const compas_b200_parm* p, const char* kind, long long s0, long long s1, long long s2) {
    int dev = 0;
    cudaGetDevice(&dev);
    return std::to_string(dev) + "/" + std::to_string(p->physics) + "/" + std::to_string(p->dim) + "/" +
           std::to_string(p->nphase) + "/" + std::to_string(p->id_limiter) + "/" + std::to_string(p->precision) +
           "/" + kind + "/" + std::to_string(s0) + "x" + std::to_string(s1) + "x" + std::to_string(s2);
}

static bool tune_lookup(const std::string& key, TuneChoice* c) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it == g_tune_cache.end()) return false;
    *c = it->second;
    return true;
}

static void tune_store(const std::string& key, const TuneChoice& c) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = c;
}

// Times launch(shape, order, tma) for every candidate (one warm-up, then `reps` timed launches) on st
// and returns the fastest; tma runs over 0 .. ntma-1. Synchronises st.
template <class F>
static int tune_candidates(F&& launch, cudaStream_t st, int reps, TuneChoice* best, int ntma = 1) {
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(COMPAS_B200_ECUDA, "event create");
    }
    int rc = COMPAS_B200_OK;
    best->ms = 3.0e38f;
    for (int sh = 0; sh < kShapes && !rc; ++sh)
        for (int od = 0; od < kOrders * ntma && !rc; ++od) {
            const int o = od % kOrders, tm = od / kOrders;
            if ((rc = launch(sh, o, tm))) break;
            cudaEventRecord(e0, st);
            for (int r = 0; r < reps && !rc; ++r) rc = launch(sh, o, tm);
            cudaEventRecord(e1, st);
            if (rc) break;
            cudaError_t e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                rc = fail(COMPAS_B200_ECUDA, std::string("autotune timing: ") + cudaGetErrorString(e));
                break;
            }
            ms /= reps;
            if (ms < best->ms) {
                best->shape = sh;
                best->order = o;
                best->tma = tm;
                best->ms = ms;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// The tuned launch shape / tile order of a single box of this size, if a level has tuned it in this
// process (the drop-in entry points reuse it; they never time anything themselves).
static int cached_shape(const compas_b200_parm* p, const compas_b200_geom* g, StageArgs& a) {
    if (!p->autotune) return 0;
    TuneChoice c;
    if (!tune_lookup(tune_key(p, "box", g->n[0], g->n[1], p->dim == 3 ? g->n[2] : 1), &c)) return 0;
    a.order = c.order;
    return c.shape;
}

// ------------------------------------------------------------------------------------------------
// TMA tensor maps of a padded state array for the halo-slab staging of the 3D mixed stage kernel
// (tma.cuh). Encoded with the driver's cuTensorMapEncodeTiled (looked up once through the runtime):
// dims {PX, PY, PZ, N} of FP64, boxes 10 x 3 x 8 x N (y slabs) and 10 x 8 x 3 x N (z slabs). The
// slab boxes start at an even x index (16-byte boundary) and at non-negative y and z. Returns false
// (maps not valid; the kernel then loads the slabs itself) where a rule does not hold: the row
// stride must be a multiple of 16 bytes (PX even), the array 16-byte aligned, 3D, ng >= 3.
// ------------------------------------------------------------------------------------------------
static bool tma_wanted(const compas_b200_parm* p) {
    return p->tma && p->dim == 3 && p->precision == 1 && !p->thinc &&
           (p->physics == COMPAS_B200_FIVEEQS || p->physics == COMPAS_B200_SIXEQS);
}

static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    std::lock_guard<std::mutex> lock(mu);
    if (!tried) {
        tried = true;
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
        else
            cudaGetLastError();
    }
    return fn;
}

static bool make_tma_maps(const compas_b200_parm* p, const compas_b200_geom* geo, const double* U, TmaMaps* out) {
    std::memset(out, 0, sizeof(*out));
    if (!tma_wanted(p) || !U) return false;
    const Grid g = make_grid(p, geo);
    if (g.ng < 3 || (g.px % 2) != 0 || (reinterpret_cast<uintptr_t>(U) % 16) != 0) return false;
    if (g.px > (1LL << 31) || g.pxy / g.px > (1LL << 31) || g.S / g.pxy > (1LL << 31)) return false;
    auto enc = tma_encoder();
    if (!enc) return false;
    const int N = nstate(p);
    const cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)(g.pxy / g.px), (cuuint64_t)(g.S / g.pxy),
                                (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)g.px * 8, (cuuint64_t)g.pxy * 8, (cuuint64_t)g.S * 8};
    const cuuint32_t box_y[4] = {(cuuint32_t)kTmaBoxX, 3, (cuuint32_t)kTile3, (cuuint32_t)N};
    const cuuint32_t box_z[4] = {(cuuint32_t)kTmaBoxX, (cuuint32_t)kTile3, 3, (cuuint32_t)N};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    void* base = const_cast<double*>(U);
    CUresult r1 = enc(&out->y, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box_y, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CUresult r2 = enc(&out->z, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box_z, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    out->valid = (r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS) ? 1 : 0;
    return out->valid != 0;
}

static StageArgs base_args(const compas_b200_parm* p, const compas_b200_geom* g) {
    StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid(p, g);
    a.e = make_eos(p);
    a.id_k = p->source_term;
    a.relax = (p->physics == COMPAS_B200_SIXEQS || p->physics == COMPAS_B200_SIXEQS_IE_NPHASE) ? p->relaxation : 0;
    a.riemann = p->id_riemann;
    a.trace = p->relax_trace;
    a.pf_phasic = (p->pf_phase2flux == 0);
    a.muscl = p->id_weno ? (p->id_limiter == 3 ? 10 : (p->id_limiter == 4 ? 11 : -1)) : p->id_limiter;
    a.pf_hll = (p->pf_flux == 1);
    a.thinc.use_normal = p->thinc_use_normal;
    a.thinc.eps = p->thinc_eps;
    a.thinc.beta = p->thinc_beta;
    a.thinc.thr = p->thinc_normal_threshold;
    return a;
}

// ------------------------------------------------------------------------------------------------
// Allocation-free RK3 step: the two intermediate stage states and the step's dt live in this
// file-scope device array instead of memory the library or the caller allocates. It is created with
// the module on every GPU that loads the library and held until the process exits.
// ------------------------------------------------------------------------------------------------
constexpr long long kNoAllocStateBytes = 16LL << 20;       // largest state array (with ghosts) accepted
constexpr long long kNoAllocHeadBytes = 256;               // dt of the step
constexpr long long kNoAllocBytes = kNoAllocHeadBytes + 2 * kNoAllocStateBytes;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

__global__ void noalloc_set_dt_kernel(double* dt_slot, double dt) { *dt_slot = dt; }

// Device address of g_noalloc_scratch on the current device, looked up once per device and kept
// for the life of the process (a cudaDeviceReset of that device invalidates it).
static int noalloc_scratch(unsigned char** out) {
    static std::mutex mu;
    static unsigned char* addr[128] = {nullptr};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return fail(COMPAS_B200_EARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(COMPAS_B200_ECUDA, std::string("cudaGetSymbolAddress of the scratch array: ") +
                                               cudaGetErrorString(e));
        addr[dev] = static_cast<unsigned char*>(ptr);
    }
    *out = addr[dev];
    return COMPAS_B200_OK;
}

// ------------------------------------------------------------------------------------------------
// Bound-preserving right-hand side (FiniteVolume.ID_Bound = 1, FIVEEQS): launch helpers of the face
// pass and the stage update of bound.cuh, and the work arrays of a level.
// ------------------------------------------------------------------------------------------------
// Quadrature weight of the limiters: 1/12 with WENO5 / WENO5B (ID_Poly 4), 1/6 otherwise (MUSCLBP's
// fixed weight; WENO3 / WENO3B run WENO5BP with ID_Poly 2), FiniteVolume_Parameter.H:60-141.
static double bp_limiter_weight(const compas_b200_parm* p) {
    return (p->id_weno && p->id_limiter >= 5) ? 1.0 / 12.0 : 1.0 / 6.0;
}
// Quadrature_Weight of the CFL speed (FiniteVolume_Parameter.H:161-173): ID_Poly 0 (GODUNOV) 1,
// 2 (MUSCL family and WENO3 / WENO3B under ID_Bound) 1/6, 4 (WENO5 / WENO5B) 1/12.
static double bp_cfl_weight(const compas_b200_parm* p) {
    if (!p->id_weno && p->id_limiter == 0) return 1.0;
    return (p->id_weno && p->id_limiter >= 5) ? 1.0 / 12.0 : 1.0 / 6.0;
}

static long long bp_face_count(const compas_b200_geom* g, int D, int d) {
    long long c = 1;
    for (int e = 0; e < D; ++e) c *= (long long)g->n[e] + (e == d);
    return c;
}

static BpFaceArgs bp_face_args(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, int id_lambda) {
    BpFaceArgs a;
    std::memset(&a, 0, sizeof(a));
    a.U = U;
    a.g = make_grid(p, g);
    a.e = make_eos(p);
    a.D = p->dim;
    a.physics = p->physics;
    a.nphase = p->nphase;
    a.weno = p->id_weno;
    a.lim = p->id_weno ? 0 : p->id_limiter;
    a.id_k = p->source_term;
    a.id_lambda = id_lambda;
    a.wb = bp_limiter_weight(p);
    a.qw = bp_cfl_weight(p);
    a.which = COMPAS_B200_FACES_ALL;
    long long tot = 0;
    for (int d = 0; d < 3; ++d) {
        a.dx[d] = g->dx[d];
        a.area[d] = 1.0;
        a.off[d] = tot;
        if (d < p->dim) tot += bp_face_count(g, p->dim, d);
    }
    a.off[3] = tot;
    return a;
}

static int launch_bp_faces(const BpFaceArgs& a, cudaStream_t st) {
    CUDA_TRY(launch_bp_faces_model(a, st));
    return COMPAS_B200_OK;
}

static BpUpdateArgs bp_update_args(const compas_b200_parm* p, const compas_b200_geom* g) {
    BpUpdateArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid(p, g);
    a.e = make_eos(p);
    a.D = p->dim;
    a.physics = p->physics;
    a.nphase = p->nphase;
    a.id_k = p->source_term;
    for (int d = 0; d < 3; ++d) a.dx[d] = g->dx[d];
    return a;
}

static int launch_bp_update(const BpUpdateArgs& a, cudaStream_t st) {
    CUDA_TRY(launch_bp_update_model(a, st));
    return COMPAS_B200_OK;
}

// Face arrays of one box: N fluxes and the normal face velocity per direction, one allocation.
struct BpFaces {
    double* base = nullptr;
    double* F[3] = {nullptr, nullptr, nullptr};
    double* V[3] = {nullptr, nullptr, nullptr};
};
static long long bp_faces_bytes(const compas_b200_parm* p, const compas_b200_geom* g) {
    long long b = 0;
    for (int d = 0; d < p->dim; ++d) b += bp_face_count(g, p->dim, d) * (nstate(p) + 1);
    return b * (long long)sizeof(double);
}
static void bp_faces_carve(const compas_b200_parm* p, const compas_b200_geom* g, double* base, BpFaces* f) {
    f->base = base;
    double* q = base;
    for (int d = 0; d < p->dim; ++d) {
        const long long c = bp_face_count(g, p->dim, d);
        f->F[d] = q;
        q += c * nstate(p);
        f->V[d] = q;
        q += c;
    }
}

// The face pass and the update of one stage (mode kModeStage or kModeDudt) of a ghost-filled Us.
static int bp_stage(const compas_b200_parm* p, const compas_b200_geom* g, const BpFaces& f, const double* Us,
                    const double* U0, double* Uout, int mode, int stage, const double* dt_dev, int id_lambda,
                    const int* done, const unsigned long long* prev_eb, int nprev, unsigned long long* eb,
                    unsigned long long* cmax, unsigned int* err, cudaStream_t st) {
    BpFaceArgs fa = bp_face_args(p, g, Us, id_lambda);
    for (int d = 0; d < p->dim; ++d) {
        fa.F[d] = f.F[d];
        fa.V[d] = f.V[d];
    }
    fa.done = done;
    fa.prev_eb = prev_eb;
    fa.nprev = nprev;
    fa.cmax = cmax;
    fa.err = err;
    int rc = launch_bp_faces(fa, st);
    if (rc) return rc;
    BpUpdateArgs ua = bp_update_args(p, g);
    ua.Us = Us;
    ua.U0 = U0;
    ua.Uout = Uout;
    ua.mode = mode;
    ua.stage = stage;
    ua.dt = dt_dev;
    for (int d = 0; d < p->dim; ++d) {
        ua.F[d] = f.F[d];
        ua.V[d] = f.V[d];
    }
    ua.done = done;
    ua.prev_eb = prev_eb;
    ua.nprev = nprev;
    ua.eb = eb;
    ua.err = err;
    return launch_bp_update(ua, st);
}

// Right-hand side or one stage through the drop-in entry points: face arrays from the stream-ordered
// allocator, released on the same stream.
static int bp_entry(const compas_b200_parm* p, const compas_b200_geom* g, const double* Us, const double* U0,
                    double* Uout, int mode, int stage, const double* dt_dev, double* cmax_dev, unsigned int* err_dev,
                    cudaStream_t st) {
    compas_b200_geom gg = *g;
    if (p->dim == 2) gg.n[2] = 1;
    void* base = nullptr;
    CUDA_TRY(cudaMallocAsync(&base, (size_t)bp_faces_bytes(p, &gg), st));
    BpFaces f;
    bp_faces_carve(p, &gg, static_cast<double*>(base), &f);
    const int rc = bp_stage(p, &gg, f, Us, U0, Uout, mode, stage, dt_dev, p->id_lambda, nullptr, nullptr, 0, nullptr,
                            reinterpret_cast<unsigned long long*>(cmax_dev), err_dev, st);
    const cudaError_t e = cudaFreeAsync(base, st);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("face scratch release: ") + cudaGetErrorString(e));
    return COMPAS_B200_OK;
}

// Work arrays of a bound-preserving level: the state at the start of the step (a step that is taken
// again starts from it), the face arrays, and the three stages' energy-bound keys.
struct BpLevel {
    double* Usave = nullptr;
    BpFaces faces;
    unsigned long long* eb = nullptr;
};

static void bp_destroy(BpLevel* b) {
    if (!b) return;
    cudaFree(b->Usave);
    cudaFree(b->faces.base);
    cudaFree(b->eb);
    delete b;
}

static int bp_create(const compas_b200_parm* p, const compas_b200_geom* g, long long state_bytes, BpLevel** out) {
    auto* b = new BpLevel();
    void* base = nullptr;
    cudaError_t e = cudaMalloc(&b->Usave, state_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&base, bp_faces_bytes(p, g));
    if (e == cudaSuccess) bp_faces_carve(p, g, static_cast<double*>(base), &b->faces);
    if (e == cudaSuccess) e = cudaMalloc(&b->eb, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        if (!b->faces.base) cudaFree(base);
        bp_destroy(b);
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? COMPAS_B200_ENOMEM : COMPAS_B200_ECUDA,
                    std::string("bound-preserving work arrays: ") + cudaGetErrorString(e));
    }
    *out = b;
    return COMPAS_B200_OK;
}

// The ordered key of the smallest energy bound (bp_min_kernel) back to a double.
__global__ void bp_key_to_double_kernel(const unsigned long long* key, double* out) {
    const unsigned long long k = *key;
    if (k == ~0ull) {
        *out = __longlong_as_double(0x7ff0000000000000ll);  // +inf: no finite value
        return;
    }
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    *out = __longlong_as_double((long long)b);
}

}  // namespace compas

#include "batch.cuh"
#include "amr.cuh"
#include "tagging.cuh"

// ================================================================================================
// C ABI
// ================================================================================================
using namespace compas;

struct compas_b200_level {
    compas_b200_parm p;
    compas_b200_geom g;
    double* U = nullptr;   // state U^n (in place across steps)
    double* U1 = nullptr;  // stage buffers
    double* U2 = nullptr;
    StepCtl* ctl = nullptr;
    double* dts = nullptr;
    int dts_cap = 0;
    long long bytes = 0;
    long long launches = 0;
    bool need_init = true;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    compas::PfLevel* pf = nullptr;  // Phase-Field work arrays (PhaseField.phase_field = 1)
    long long pf_substeps = 0;
    compas::PfInfo pf_last{};       // counters of the last Phase-Field step
    compas::BpLevel* bp = nullptr;  // bound-preserving work arrays (FiniteVolume.ID_Bound = 1)
    long long bp_restarts = 0;
    int shape = 0, order = 0;       // stage-kernel launch shape and tile order (autotuner or forced)
    bool tuned = false, forced = false;
    compas::TmaMaps maps[3];        // TMA maps of U, U1, U2 (3D mixed form; valid = 0 otherwise)
    bool use_tma = false;           // stage with the maps (compas_b200.tma = 1; the autotuner may turn it off)
    // host-buffer steps (compas_b200_level_step_host): copy streams and the events that order the slabs
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_start = nullptr, ev_done = nullptr;
    cudaEvent_t ev_in[64] = {}, ev_out[64] = {};
};

namespace compas {

static void set_pf_args(StageArgs& a, const double* const* gq) {
    for (int d = 0; d < 3; ++d) a.gq[d] = gq[d];
}

__global__ void set_scalar_kernel(double* slot, double v) { *slot = v; }

// The sub-stepped Phase-Field TVD-RK3 advance over dt with fixed face gradients
// (PhaseField_Evolve :546-592, PhaseField_ComputeDt :2036-2098, PhaseField_ThirdOrderSSPRK :2619-2752).
// U is advanced in place with U1, U2 as stage buffers. Returns the sub-steps through *steps.
static int pf_advance(const compas_b200_parm* p, const compas_b200_geom* g, double* U, double* U1, double* U2,
                      const double* const* gq, double* dt_slot, double dt, double gmax, unsigned int* err_dev,
                      cudaStream_t st, int* steps, long long* launches) {
    double dxmin = g->dx[0];
    for (int d = 1; d < p->dim; ++d) dxmin = std::min(dxmin, g->dx[d]);
    StageArgs a = base_args(p, g);
    a.mode = kModeStage;
    a.dt = dt_slot;
    a.err = err_dev;
    set_pf_args(a, gq);
    double* bufs_in[3] = {U, U1, U2};
    double* bufs_out[3] = {U1, U2, U};
    double pft = 0.0, pfdt = 0.0;
    int n = 0, rc;
    for (int s = 0; s < p->pf_max_step && pft < dt; ++s) {
        double tmp = p->pf_cfl * dxmin / (gmax + 1.0e-14);
        if (pft == 0.0) pfdt = tmp;
        if (p->change_limiter && pfdt > 0.0) tmp = std::min(tmp, 1.1 * pfdt);
        double d0 = tmp;
        const double eps = 1.0e-3 * d0;
        if (pft + d0 > dt - eps) d0 = dt - pft;
        pfdt = d0;
        set_scalar_kernel<<<1, 1, 0, st>>>(dt_slot, pfdt);
        CUDA_TRY(cudaGetLastError());
        for (int k = 0; k < 3; ++k) {
            if ((rc = launch_fill(p, g, bufs_in[k], st))) return rc;
            a.stage = k;
            a.Us = bufs_in[k];
            a.U0 = U;
            a.Uout = bufs_out[k];
            if ((rc = launch_stage(p, a, st, 1))) return rc;
        }
        *launches += 7;
        pft += pfdt;
        ++n;
        if (pft >= dt - 1.0e-6 * dt) break;
    }
    *steps = n;
    return COMPAS_B200_OK;
}

}  // namespace compas

extern "C" {

const char* compas_b200_last_error(void) { return g_last_error.c_str(); }

int compas_b200_parm_init(compas_b200_parm* p, int physics, int dim) {
    return compas_b200_parm_init_nphase(p, physics, dim, 2);
}

int compas_b200_parm_init_nphase(compas_b200_parm* p, int physics, int dim, int nphase) {
    if (!p) return fail(COMPAS_B200_EARG, "null parm");
    std::memset(p, 0, sizeof(*p));
    p->physics = physics;
    p->dim = dim;
    p->nphase = nphase;
    p->eos = 1;
    p->gamma_1 = 1.4;
    p->gamma_2 = 1.4;
    for (int k = 0; k < kMaxPhases; ++k) p->gamma_k[k] = 1.4;
    p->id_limiter = 5;
    p->id_weno = 1;
    p->num_grow = 3;
    p->thinc = 0;
    p->thinc_use_normal = 1;
    p->thinc_eps = 1.0e-4;
    p->thinc_beta = 2.3;
    p->thinc_normal_threshold = 0.25;
    p->id_riemann = 2;
    p->cfl = 0.4;
    p->change_limiter = 1;
    // PhaseField_Parameter defaults (include/Physics_PhaseField/PhaseField_Parameter.H:27-50): the
    // inputs default mechanism is CAC-Adv (:52)
    p->pf_mechanism = 1;
    // PhaseField.ID_FluxPhase2Flux: the mixture formulation, except for the six-equation model whose
    // Parm.H selects the phasic one (exec/_Tests/Advection/prob/Parm.H:48-50)
    p->pf_phase2flux = (physics == COMPAS_B200_SIXEQS) ? 0 : 1;
    p->pf_eta_factor = 2.0;
    p->pf_eta_multiplier = 1.0;
    p->pf_cfl = 0.4;
    p->pf_max_step = 1000000;
    p->pf_tol_rel = 1.0e-10;
    p->autotune = 1;
    p->tma = 1;
    p->cv_1 = 1.0;
    p->cv_2 = 1.0;
    p->id_lambda = 1;
    if (physics != COMPAS_B200_FIVEEQS && physics != COMPAS_B200_SIXEQS && physics != COMPAS_B200_FIVEEQS_NPHASE &&
        physics != COMPAS_B200_SIXEQS_IE_NPHASE)
        return fail(COMPAS_B200_EARG, "physics must be FIVEEQS (555), SIXEQS (666), FIVEEQS_NPHASE (55501) or "
                                      "SIXEQS_IE_NPHASE (66601)");
    if (dim != 2 && dim != 3) return fail(COMPAS_B200_EARG, "dim must be 2 or 3");
    if (nphase_model(physics) && (nphase < 2 || nphase > kMaxPhases))
        return fail(COMPAS_B200_EARG, "the N-phase models: nphase must be in [2, " + std::to_string(kMaxPhases) + "]");
    if (!nphase_model(physics) && nphase != 2)
        return fail(COMPAS_B200_EARG, "the two-phase models have nphase = 2");
    return compas_b200_parm_finalize(p);
}

static bool parse_double(const char* v, double* out) {
    char* end = nullptr;
    const double x = std::strtod(v, &end);
    if (end == v) return false;
    while (*end == ' ') ++end;
    if (*end) return false;
    *out = x;
    return true;
}

static bool parse_int(const char* v, int* out) {
    char* end = nullptr;
    const long x = std::strtol(v, &end, 10);
    if (end == v) return false;
    while (*end == ' ') ++end;
    if (*end) return false;
    *out = (int)x;
    return true;
}

int compas_b200_parm_set(compas_b200_parm* p, const char* key, const char* value) {
    if (!p || !key || !value) return fail(COMPAS_B200_EARG, "null argument");
    const std::string k(key), v(value);
    auto bad = [&](const std::string& valid) {
        return fail(COMPAS_B200_EARG, k + " = '" + v + "' is not recognized. Valid values are " + valid + ".");
    };
    double x;
    int ix;
    if (k == "FiniteVolume.Scheme") {
        // include/Operators_FV/FiniteVolume_Parameter.H:51-147
        if (v == "WENO5") { p->id_limiter = 5; p->id_weno = 1; p->num_grow = 3; return 0; }
        if (v == "WENO5B") { p->id_limiter = 6; p->id_weno = 1; p->num_grow = 3; return 0; }
        if (v == "GODUNOV") { p->id_limiter = 0; p->id_weno = 0; p->num_grow = 1; return 0; }
        if (v == "MUSCL" || v == "MUSCL-Minmod") { p->id_limiter = 1; p->id_weno = 0; p->num_grow = 2; return 0; }
        if (v == "MUSCL-vanLeer") { p->id_limiter = 2; p->id_weno = 0; p->num_grow = 2; return 0; }
        if (v == "MUSCL-Superbee") { p->id_limiter = 3; p->id_weno = 0; p->num_grow = 2; return 0; }
        if (v == "MUSCL-MC") { p->id_limiter = 4; p->id_weno = 0; p->num_grow = 2; return 0; }
        if (v == "WENO3") { p->id_limiter = 3; p->id_weno = 1; p->num_grow = 2; return 0; }
        if (v == "WENO3B") { p->id_limiter = 4; p->id_weno = 1; p->num_grow = 2; return 0; }
        return bad("GODUNOV, MUSCL, MUSCL-Minmod, MUSCL-vanLeer, MUSCL-Superbee, MUSCL-MC, WENO3, WENO3B, WENO5, WENO5B");
    }
    if (k == "FiniteVolume.THINC") { if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1"); p->thinc = ix; return 0; }
    if (k == "FiniteVolume.THINC.UseNormal") { if (!parse_int(value, &ix)) return bad("an integer"); p->thinc_use_normal = ix; return 0; }
    if (k == "FiniteVolume.THINC.EPS") { if (!parse_double(value, &x)) return bad("a number"); p->thinc_eps = x; return 0; }
    if (k == "FiniteVolume.THINC.Beta") { if (!parse_double(value, &x)) return bad("a number"); p->thinc_beta = x; return 0; }
    if (k == "FiniteVolume.THINC.NormalThreshold") { if (!parse_double(value, &x)) return bad("a number"); p->thinc_normal_threshold = x; return 0; }
    if (k == "FiniteVolume.ID_Bound") {
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1");
        p->id_bound = ix;
        return 0;
    }
    if (k == "Physics.RiemannSolver") {
        // source/Class_Compressible_PhaseField.cpp:92-111
        if (v == "HLLC") { p->id_riemann = 2; return 0; }
        if (v == "LLF" || v == "HLL") { p->id_riemann = (v == "LLF") ? 0 : 1; return 0; }
        return bad("LLF, HLL, HLLC");
    }
    if (k == "Physics.source_term") {
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return fail(COMPAS_B200_EARG, "Physics.source_term must be 0 or 1.");
        p->source_term = ix;
        return 0;
    }
    if (k == "Physics.pressure_relaxation") { if (!parse_int(value, &ix)) return bad("0, 1"); p->relaxation = ix ? 1 : 0; return 0; }
    if (k == "Physics.pressure_relaxation_trace") {
        if (!parse_double(value, &x) || x < 0.0 || x >= 1.0)
            return fail(COMPAS_B200_EARG, "Physics.pressure_relaxation_trace must be in [0, 1).");
        p->relax_trace = x;
        return 0;
    }
    if (k == "prob.EOS.EOS") {
        if (!parse_int(value, &ix) || (ix != 0 && ix != 1 && ix != 3))
            return fail(COMPAS_B200_EARG, "prob.EOS.EOS = " + v + " is not recognized. Valid values are 0 (ideal gas), "
                                          "1 (stiffened gas), 3 (Noble-Abel stiffened gas); 2 (Mie-Gruneisen) is outside "
                                          "this engine's hot path.");
        p->eos = ix;
        return 0;
    }
    if (nphase_model(p->physics)) {
        // per-phase lists (source/Parm.cpp:66-92): exactly NPHASE values
        struct LKey { const char* name; double* dst; };
        const LKey lkeys[] = {{"prob.EOS.gamma", p->gamma_k}, {"prob.EOS.pinf", p->pinf_k},
                              {"prob.EOS.b", p->b_k}, {"prob.EOS.q", p->q_k}};
        for (const auto& lk : lkeys)
            if (k == lk.name) {
                double vals[kMaxPhases];
                int cnt = 0;
                const char* c = value;
                while (true) {
                    while (*c == ' ' || *c == '\t' || *c == ',') ++c;
                    if (!*c) break;
                    char* end = nullptr;
                    const double x1 = std::strtod(c, &end);
                    if (end == c) return bad("a list of numbers");
                    if (cnt < kMaxPhases) vals[cnt] = x1;
                    ++cnt;
                    c = end;
                }
                if (cnt != p->nphase)
                    return fail(COMPAS_B200_EARG, k + " has " + std::to_string(cnt) + " values, but NPHASE = " +
                                                      std::to_string(p->nphase) + " needs one value per phase.");
                for (int i = 0; i < cnt; ++i) lk.dst[i] = vals[i];
                return 0;
            }
    }
    struct DKey { const char* name; double* dst; };
    const DKey dkeys[] = {{"prob.EOS.gamma_1", &p->gamma_1}, {"prob.EOS.gamma_2", &p->gamma_2},
                          {"prob.EOS.pinf_1", &p->pinf_1},   {"prob.EOS.pinf_2", &p->pinf_2},
                          {"prob.EOS.b_1", &p->b_1},         {"prob.EOS.b_2", &p->b_2},
                          {"prob.EOS.q_1", &p->q_1},         {"prob.EOS.q_2", &p->q_2},
                          {"prob.EOS.cv_1", &p->cv_1},       {"prob.EOS.cv_2", &p->cv_2},
                          {"run.cfl", &p->cfl}};
    for (const auto& dk : dkeys)
        if (k == dk.name) {
            if (!parse_double(value, &x)) return bad("a number");
            *dk.dst = x;
            return 0;
        }
    if (k == "compas_b200.tma") {
        // this engine's own key: stage the 3D mixed form's halo slabs by TMA (1) or plain loads (0)
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1");
        p->tma = ix;
        return 0;
    }
    if (k == "compas_b200.autotune") {
        // this engine's own key: pick the stage kernel's launch shape and tile order by timing
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1");
        p->autotune = ix;
        return 0;
    }
    if (k == "compas_b200.precision") {
        // this engine's own key (no reference counterpart): the arithmetic of the bulk of the RHS
        if (v == "fp64") { p->precision = 0; return 0; }
        if (v == "mixed") { p->precision = 1; return 0; }
        return bad("fp64, mixed");
    }
    if (k == "PhaseField.Mechanism") {
        // include/Physics_PhaseField/PhaseField_Parameter.H:66-115
        if (v == "CAC-Adv") { p->pf_mechanism = 1; return 0; }
        if (v == "ACDI") { p->pf_mechanism = 3; return 0; }
        if (v == "CAC-Adv-NormalFace" || v == "CAC-VanDerWaals" || v == "CDI" || v == "CDI-NormalFace" ||
            v == "CDI-CompressionInterpolation" || v == "ACDI-NormalFace" || v == "CH-Adv" || v == "CH-Adv-NormalFace" ||
            v == "CH-VanDerWaals")
            return fail(COMPAS_B200_EUNSUPPORTED, k + " = " + v + " is a valid reference mechanism outside this engine "
                                                  "(CAC-Adv, ACDI)");
        return bad("CAC-Adv, CAC-Adv-NormalFace, CAC-VanDerWaals, CDI, CDI-NormalFace, CDI-CompressionInterpolation, "
                   "ACDI, ACDI-NormalFace, CH-Adv, CH-Adv-NormalFace, CH-VanDerWaals");
    }
    if (k == "PhaseField.phase_field") { if (!parse_int(value, &ix)) return bad("0, 1"); p->phase_field = ix ? 1 : 0; return 0; }
    if (k == "PhaseField.ID_ExplicitRC") { if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1"); p->pf_explicit_rc = ix; return 0; }
    if (k == "PhaseField.ID_Flux") {
        // include/Physics_PhaseField/PhaseField_Parameter.H:52 (0 upwind/downwind, 1 HLL)
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1");
        p->pf_flux = ix;
        return 0;
    }
    if (k == "PhaseField.ID_FluxPhase2Flux") {
        // include/Physics_PhaseField/PhaseField_Parameter.H:53 (0 phasic, 1 mixture formulation)
        if (!parse_int(value, &ix) || ix < 0 || ix > 1) return bad("0, 1");
        p->pf_phase2flux = ix;
        return 0;
    }
    if (k == "PhaseField.max_step") { if (!parse_int(value, &ix)) return bad("an integer"); p->pf_max_step = ix; return 0; }
    {
        struct PKey { const char* name; double* dst; };
        const PKey pkeys[] = {{"PhaseField.Lambda", &p->pf_lambda}, {"PhaseField.Eta", &p->pf_eta},
                              {"PhaseField.Eta_Factor", &p->pf_eta_factor},
                              {"PhaseField.Eta_Multiplier", &p->pf_eta_multiplier},
                              {"PhaseField.cfl", &p->pf_cfl}, {"LinearSystem.tol_rel", &p->pf_tol_rel}};
        for (const auto& pk : pkeys)
            if (k == pk.name) {
                if (!parse_double(value, &x)) return bad("a number");
                *pk.dst = x;
                return 0;
            }
    }
    // options the engine runs only at their reference defaults (PhaseField_Parameter.H:40-48)
    {
        struct OKey { const char* name; int only; };
        const OKey okeys[] = {{"PhaseField.ID_Weight", 0}, {"PhaseField.ID_Potential", 0},
                              {"PhaseField.ID_DegenerateMobility", 0}, {"PhaseField.ID_Formulation", 1},
                              {"PhaseField.Switch_Step", 0}};
        for (const auto& ok : okeys)
            if (k == ok.name) {
                if (!parse_int(value, &ix)) return bad("an integer");
                if (ix != ok.only)
                    return fail(COMPAS_B200_EUNSUPPORTED, k + " = " + v + ": this engine runs the reference default " +
                                                              std::to_string(ok.only));
                return 0;
            }
    }
    if (k == "amr.Interpolater") {
        // source/COMPAS.cpp:1217-1221
        if (v == "lincc_interp") { p->amr_interp = 0; return 0; }
        if (v == "pc_interp") { p->amr_interp = 1; return 0; }
        if (v == "quartic_interp")
            return fail(COMPAS_B200_EUNSUPPORTED, "amr.Interpolater = quartic_interp is not in this engine");
        return bad("pc_interp, lincc_interp, quartic_interp");
    }
    if (k == "run.timestep_change_limiter") { if (!parse_int(value, &ix)) return bad("0, 1"); p->change_limiter = ix ? 1 : 0; return 0; }
    return fail(COMPAS_B200_EARG, "unknown inputs key '" + k + "'");
}

int compas_b200_parm_finalize(compas_b200_parm* p) {
    if (!p) return fail(COMPAS_B200_EARG, "null parm");
    if (nphase_model(p->physics)) {
        // source/Parm.cpp:185-253 (FIVEEQS_NPHASE), :364-446 (SIXEQS_IE_NPHASE, the same coefficients)
        const int np = p->nphase;
        if (np < 2 || np > kMaxPhases) return fail(COMPAS_B200_EARG, "the N-phase models: nphase out of range");
        for (int k = 0; k < np; ++k) {
            if (!(p->gamma_k[k] > 1.0))
                return fail(COMPAS_B200_EARG, "prob.EOS.EOS requires gamma > 1, but prob.EOS.gamma[" +
                                                  std::to_string(k) + "] is " + std::to_string(p->gamma_k[k]));
            const double g = p->gamma_k[k];
            p->Ak[k] = 1. / (g - 1.);
            if (p->eos == 0) {
                p->Bk[k] = 0.0; p->Ck[k] = 0.0; p->Dk[k] = 0.0;
            } else if (p->eos == 1) {
                p->Bk[k] = g * p->pinf_k[k] / (g - 1.);
                p->Ck[k] = 0.0; p->Dk[k] = 0.0;
            } else if (p->eos == 3) {
                if (p->b_k[k] < 0.0) return fail(COMPAS_B200_EARG, "prob.EOS.b must be >= 0");
                p->Bk[k] = g * p->pinf_k[k] / (g - 1.);
                p->Ck[k] = p->b_k[k];
                p->Dk[k] = p->q_k[k];
            } else {
                return fail(COMPAS_B200_EARG, "prob.EOS.EOS must be 0, 1 or 3");
            }
        }
        for (int k = np; k < kMaxPhases; ++k) {
            p->Ak[k] = 1.0; p->Bk[k] = 0.0; p->Ck[k] = 0.0; p->Dk[k] = 0.0;
        }
        // the two-phase fields stay valid (A = 1/(1.4 - 1)) so that shared code never divides by 0
        p->A1 = p->Ak[0]; p->A2 = p->Ak[1];
        return COMPAS_B200_OK;
    }
    // source/Parm.cpp:101-188
    if (!(p->gamma_1 > 1.0) || !(p->gamma_2 > 1.0))
        return fail(COMPAS_B200_EARG, "prob.EOS.EOS requires gamma > 1 for both phases");
    p->A1 = 1. / (p->gamma_1 - 1.);
    p->A2 = 1. / (p->gamma_2 - 1.);
    if (p->eos == 0) {
        p->B1 = 0.; p->B2 = 0.; p->C1 = 0.; p->C2 = 0.; p->D1 = 0.; p->D2 = 0.;
    } else if (p->eos == 1) {
        p->B1 = p->gamma_1 * p->pinf_1 / (p->gamma_1 - 1.);
        p->B2 = p->gamma_2 * p->pinf_2 / (p->gamma_2 - 1.);
        p->C1 = 0.; p->C2 = 0.; p->D1 = 0.; p->D2 = 0.;
    } else if (p->eos == 3) {
        if (p->b_1 < 0.0 || p->b_2 < 0.0) return fail(COMPAS_B200_EARG, "prob.EOS.b_k must be >= 0");
        p->B1 = p->gamma_1 * p->pinf_1 / (p->gamma_1 - 1.);
        p->B2 = p->gamma_2 * p->pinf_2 / (p->gamma_2 - 1.);
        p->C1 = p->b_1; p->C2 = p->b_2; p->D1 = p->q_1; p->D2 = p->q_2;
    } else {
        return fail(COMPAS_B200_EARG, "prob.EOS.EOS must be 0, 1 or 3");
    }
    return COMPAS_B200_OK;
}

long long compas_b200_state_bytes(const compas_b200_parm* p, const compas_b200_geom* g) {
    if (!p || !g) return 0;
    const Grid G = make_grid(p, g);
    return G.S * (long long)nstate(p) * (long long)sizeof(double);
}

int compas_b200_fill_boundary(const compas_b200_parm* p, const compas_b200_geom* g, double* U, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U) return fail(COMPAS_B200_EARG, "null state");
    return launch_fill(p, g, U, (cudaStream_t)stream);
}

int compas_b200_compute_dUdt(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double* dUdt,
                             double* cmax_dev, unsigned int* err_dev, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U || !dUdt) return fail(COMPAS_B200_EARG, "null state");
    if (p->id_bound)
        return bp_entry(p, g, U, nullptr, dUdt, kModeDudt, 0, nullptr, cmax_dev, err_dev, (cudaStream_t)stream);
    StageArgs a = base_args(p, g);
    a.Us = U;
    a.Uout = dUdt;
    a.mode = kModeDudt;
    a.cmax = reinterpret_cast<unsigned long long*>(cmax_dev);
    a.err = err_dev;
    const int shape = cached_shape(p, g, a);
    return launch_stage(p, a, (cudaStream_t)stream, 0, shape);
}

int compas_b200_rk3_stage(const compas_b200_parm* p, const compas_b200_geom* g, int stage, const double* Us,
                          const double* Uold, double* Unew, const double* dt_dev, double* cmax_dev,
                          unsigned int* err_dev, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (stage < 0 || stage > 2) return fail(COMPAS_B200_EARG, "stage must be 0, 1 or 2");
    if (!Us || !Unew || !dt_dev || (stage > 0 && !Uold)) return fail(COMPAS_B200_EARG, "null argument");
    if (Us == Unew) return fail(COMPAS_B200_EARG, "Unew may not alias Us");
    if (p->id_bound)
        return bp_entry(p, g, Us, Uold, Unew, kModeStage, stage, dt_dev, cmax_dev, err_dev, (cudaStream_t)stream);
    StageArgs a = base_args(p, g);
    a.Us = Us;
    a.U0 = Uold;
    a.Uout = Unew;
    a.mode = kModeStage;
    a.stage = stage;
    a.dt = dt_dev;
    a.cmax = reinterpret_cast<unsigned long long*>(cmax_dev);
    a.err = err_dev;
    const int shape = cached_shape(p, g, a);
    return launch_stage(p, a, (cudaStream_t)stream, 0, shape);
}

int compas_b200_pf_compute_dUdt(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double* dUdt,
                                const double* gq0, const double* gq1, const double* gq2, unsigned int* err_dev,
                                void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (p->id_bound)
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field step with FiniteVolume.ID_Bound = 1 is not in this engine");
    if (nphase_model(p->physics))
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field right-hand side is the two-phase models'");
    if (!U || !dUdt || !gq0 || !gq1 || (p->dim == 3 && !gq2)) return fail(COMPAS_B200_EARG, "null argument");
    StageArgs a = base_args(p, g);
    a.Us = U;
    a.Uout = dUdt;
    a.mode = kModeDudt;
    a.err = err_dev;
    const double* gq[3] = {gq0, gq1, gq2};
    set_pf_args(a, gq);
    return launch_stage(p, a, (cudaStream_t)stream, 1);
}

int compas_b200_pf_rk3_stage(const compas_b200_parm* p, const compas_b200_geom* g, int stage, const double* Us,
                             const double* Uold, double* Unew, const double* dt_dev, const double* gq0,
                             const double* gq1, const double* gq2, unsigned int* err_dev, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (p->id_bound)
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field step with FiniteVolume.ID_Bound = 1 is not in this engine");
    if (nphase_model(p->physics))
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field right-hand side is the two-phase models'");
    if (stage < 0 || stage > 2) return fail(COMPAS_B200_EARG, "stage must be 0, 1 or 2");
    if (!Us || !Unew || !dt_dev || (stage > 0 && !Uold) || !gq0 || !gq1 || (p->dim == 3 && !gq2))
        return fail(COMPAS_B200_EARG, "null argument");
    if (Us == Unew) return fail(COMPAS_B200_EARG, "Unew may not alias Us");
    StageArgs a = base_args(p, g);
    a.Us = Us;
    a.U0 = Uold;
    a.Uout = Unew;
    a.mode = kModeStage;
    a.stage = stage;
    a.dt = dt_dev;
    a.err = err_dev;
    const double* gq[3] = {gq0, gq1, gq2};
    set_pf_args(a, gq);
    return launch_stage(p, a, (cudaStream_t)stream, 1);
}

int compas_b200_pf_grad_q(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double dt,
                          double* gq0, double* gq1, double* gq2, double* info, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (p->id_bound)
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field step with FiniteVolume.ID_Bound = 1 is not in this engine");
    if (nphase_model(p->physics))
        return fail(COMPAS_B200_EUNSUPPORTED, "the Phase-Field step is the two-phase models'");
    if (!U || !gq0 || !gq1 || (p->dim == 3 && !gq2)) return fail(COMPAS_B200_EARG, "null argument");
    if (!(dt > 0.0)) return fail(COMPAS_B200_EARG, "dt must be positive");
    compas_b200_geom gg = *g;
    if (p->dim == 2) gg.n[2] = 1;
    PfLevel* pf = nullptr;
    std::string msg;
    if ((rc = pf_create(p, &gg, &pf, &msg))) return fail(rc, msg);
    cudaStream_t st = (cudaStream_t)stream;
    PfInfo pi;
    rc = pf_grad_q(pf, p, U, dt, st, &pi, &msg);
    if (!rc) {
        double* out[3] = {gq0, gq1, gq2};
        for (int d = 0; d < p->dim && !rc; ++d) {
            const long long nf = (long long)(gg.n[0] + (d == 0)) * (gg.n[1] + (d == 1)) * (gg.n[2] + (d == 2));
            cudaError_t e = cudaMemcpyAsync(out[d], pf_gq(pf, d), sizeof(double) * nf, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) {
                rc = COMPAS_B200_ECUDA;
                msg = std::string("copy of grad Q: ") + cudaGetErrorString(e);
            }
        }
        if (!rc && cudaStreamSynchronize(st) != cudaSuccess) {
            rc = COMPAS_B200_ECUDA;
            msg = "stream synchronisation";
        }
    }
    pf_destroy(pf);
    if (rc) return fail(rc, msg);
    if (info) {
        info[0] = pi.max_v;
        info[1] = pi.mobility;
        info[2] = pi.eta;
        info[3] = pi.mech_steps;
        info[4] = pi.solve_iters;
        info[5] = pi.gmax;
        info[6] = pi.solve_res;
    }
    return COMPAS_B200_OK;
}

long long compas_b200_level_pf_substeps(const compas_b200_level* lv) { return lv ? lv->pf_substeps : 0; }

int compas_b200_level_pf_info(const compas_b200_level* lv, double* info) {
    if (!lv || !info) return fail(COMPAS_B200_EARG, "null argument");
    const PfInfo& i = lv->pf_last;
    info[0] = i.max_v;
    info[1] = i.mobility;
    info[2] = i.eta;
    info[3] = i.mech_steps;
    info[4] = i.solve_iters;
    info[5] = i.gmax;
    info[6] = i.solve_res;
    return COMPAS_B200_OK;
}

int compas_b200_relaxation(const compas_b200_parm* p, const compas_b200_geom* g, double* U, unsigned int* err_dev,
                           void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (p->physics != COMPAS_B200_SIXEQS) return COMPAS_B200_OK;
    const Grid G = make_grid(p, g);
    const long long cells = (long long)G.n[0] * G.n[1] * G.n[2];
    long long blocks = (cells + 127) / 128;
    if (blocks > 148LL * 32) blocks = 148LL * 32;
    if (p->dim == 2)
        relax_kernel<2><<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>(U, G, make_eos(p), p->relax_trace, err_dev);
    else
        relax_kernel<3><<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>(U, G, make_eos(p), p->relax_trace, err_dev);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

// One TVD-RK3 step in place on the caller's state U without allocating device memory. The two
// intermediate stage states and the device copy of dt live in g_noalloc_scratch; everything else is
// the same launches as compas_b200_rk3_stage (boundary fill, then the fused stage kernel, three times).
int compas_b200_rk3_step_noalloc(const compas_b200_parm* p, const compas_b200_geom* g, double* U, double dt,
                                 double* cmax_dev, unsigned int* err_dev, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U) return fail(COMPAS_B200_EARG, "null state");
    if (p->id_bound)
        return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1 runs on the level API (its steps may be taken "
                                              "again), not in the allocation-free step");
    if (!(dt > 0.0) || !(dt <= DBL_MAX)) return fail(COMPAS_B200_EARG, "dt must be positive and finite");
    const long long bytes = compas_b200_state_bytes(p, g);
    if (bytes > kNoAllocStateBytes)
        return fail(COMPAS_B200_EARG, "state of " + std::to_string(bytes) + " bytes exceeds the " +
                                          std::to_string(kNoAllocStateBytes) +
                                          "-byte limit of the allocation-free step; use the level API");
    unsigned char* base = nullptr;
    if ((rc = noalloc_scratch(&base))) return rc;
    double* dt_dev = reinterpret_cast<double*>(base);
    double* U1 = reinterpret_cast<double*>(base + kNoAllocHeadBytes);
    double* U2 = reinterpret_cast<double*>(base + kNoAllocHeadBytes + kNoAllocStateBytes);
    cudaStream_t st = (cudaStream_t)stream;
    // the scratch keeps the previous call's contents: dt is rewritten here, U1 and U2 are fully
    // written (valid cells by the stage kernels, ghosts by the boundary fill) before they are read
    noalloc_set_dt_kernel<<<1, 1, 0, st>>>(dt_dev, dt);
    CUDA_TRY(cudaGetLastError());
    StageArgs a = base_args(p, g);
    a.mode = kModeStage;
    a.dt = dt_dev;
    a.cmax = reinterpret_cast<unsigned long long*>(cmax_dev);
    a.err = err_dev;
    const int shape = cached_shape(p, g, a);  // a host-side cache read: allocates nothing
    double* ins[3] = {U, U1, U2};
    double* outs[3] = {U1, U2, U};
    for (int s = 0; s < 3; ++s) {
        if ((rc = launch_fill(p, g, ins[s], st))) return rc;
        a.stage = s;
        a.Us = ins[s];
        a.U0 = U;
        a.Uout = outs[s];
        if ((rc = launch_stage(p, a, st, 0, shape))) return rc;
    }
    return COMPAS_B200_OK;
}

int compas_b200_level_create(const compas_b200_parm* p, const compas_b200_geom* g, compas_b200_level** out) {
    if (!out) return fail(COMPAS_B200_EARG, "null output");
    *out = nullptr;
    int rc = check_args(p, g);
    if (rc) return rc;
    auto* lv = new compas_b200_level();
    lv->p = *p;
    lv->g = *g;
    if (p->dim == 2) lv->g.n[2] = 1;
    lv->bytes = compas_b200_state_bytes(p, g);
    lv->dts_cap = 1 << 16;
    cudaError_t e = cudaMalloc(&lv->U, lv->bytes);
    if (e == cudaSuccess) e = cudaMalloc(&lv->U1, lv->bytes);
    if (e == cudaSuccess) e = cudaMalloc(&lv->U2, lv->bytes);
    if (e == cudaSuccess) e = cudaMalloc(&lv->ctl, sizeof(StepCtl));
    if (e == cudaSuccess) e = cudaMalloc(&lv->dts, sizeof(double) * lv->dts_cap);
    if (e == cudaSuccess) e = cudaMemset(lv->ctl, 0, sizeof(StepCtl));
    if (e == cudaSuccess) e = cudaMemset(lv->U, 0, lv->bytes);
    if (e == cudaSuccess) e = cudaMemset(lv->U1, 0, lv->bytes);
    if (e == cudaSuccess) e = cudaMemset(lv->U2, 0, lv->bytes);
    if (e != cudaSuccess) {
        compas_b200_level_destroy(lv);
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? COMPAS_B200_ENOMEM : COMPAS_B200_ECUDA,
                    std::string("level allocation: ") + cudaGetErrorString(e));
    }
    make_tma_maps(p, &lv->g, lv->U, &lv->maps[0]);
    make_tma_maps(p, &lv->g, lv->U1, &lv->maps[1]);
    make_tma_maps(p, &lv->g, lv->U2, &lv->maps[2]);
    lv->use_tma = lv->maps[0].valid && lv->maps[1].valid && lv->maps[2].valid;
    if (p->id_bound && (rc = bp_create(p, &lv->g, lv->bytes, &lv->bp))) {
        compas_b200_level_destroy(lv);
        return rc;
    }
    if (p->phase_field) {
        std::string msg;
        if ((rc = pf_create(p, &lv->g, &lv->pf, &msg))) {
            compas_b200_level_destroy(lv);
            cudaGetLastError();
            return fail(rc, msg);
        }
    }
    *out = lv;
    return COMPAS_B200_OK;
}

int compas_b200_level_destroy(compas_b200_level* lv) {
    if (!lv) return COMPAS_B200_OK;
    if (lv->graph) cudaGraphExecDestroy(lv->graph);
    if (lv->h2d) {
        cudaStreamSynchronize(lv->h2d);
        cudaStreamSynchronize(lv->d2h);
        cudaStreamDestroy(lv->h2d);
        cudaStreamDestroy(lv->d2h);
        cudaEventDestroy(lv->ev_start);
        cudaEventDestroy(lv->ev_done);
        for (int c = 0; c < 64; ++c) {
            cudaEventDestroy(lv->ev_in[c]);
            cudaEventDestroy(lv->ev_out[c]);
        }
    }
    cudaFree(lv->U);
    cudaFree(lv->U1);
    cudaFree(lv->U2);
    cudaFree(lv->ctl);
    cudaFree(lv->dts);
    pf_destroy(lv->pf);
    bp_destroy(lv->bp);
    delete lv;
    return COMPAS_B200_OK;
}

double* compas_b200_level_state(compas_b200_level* lv) { return lv ? lv->U : nullptr; }

long long compas_b200_level_launches(compas_b200_level* lv) { return lv ? lv->launches : 0; }

int compas_b200_level_upload(compas_b200_level* lv, const double* src, int is_device, double t0, void* stream) {
    if (!lv || !src) return fail(COMPAS_B200_EARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(lv->U, src, lv->bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    set_time_kernel<<<1, 1, 0, st>>>(lv->ctl, t0, 0.0, 1);
    CUDA_TRY(cudaGetLastError());
    lv->launches = 1;
    lv->need_init = true;
    return COMPAS_B200_OK;
}

int compas_b200_level_set_state(compas_b200_level* lv, const double* src, int is_device, void* stream) {
    if (!lv || !src) return fail(COMPAS_B200_EARG, "null argument");
    CUDA_TRY(cudaMemcpyAsync(lv->U, src, lv->bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                             (cudaStream_t)stream));
    return COMPAS_B200_OK;
}

int compas_b200_level_download(compas_b200_level* lv, double* dst, int is_device, void* stream) {
    if (!lv || !dst) return fail(COMPAS_B200_EARG, "null argument");
    CUDA_TRY(cudaMemcpyAsync(dst, lv->U, lv->bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream));
    return COMPAS_B200_OK;
}

// Autotune the level's stage kernel on its own state (ghosts filled): a stage-0 launch with dt = 0
// into the stage buffer U1 per candidate, wave speeds and status into a scratch block.
static int tune_level(compas_b200_level* lv, cudaStream_t st) {
    const std::string key = tune_key(&lv->p, "box", lv->g.n[0], lv->g.n[1], lv->p.dim == 3 ? lv->g.n[2] : 1);
    TuneChoice c;
    if (!tune_lookup(key, &c)) {
        double* scratch = nullptr;
        CUDA_TRY(cudaMalloc(&scratch, 64));
        cudaError_t e = cudaMemsetAsync(scratch, 0, 64, st);
        if (e != cudaSuccess) {
            cudaFree(scratch);
            return fail(COMPAS_B200_ECUDA, std::string("autotune scratch: ") + cudaGetErrorString(e));
        }
        StageArgs a = base_args(&lv->p, &lv->g);
        a.mode = kModeStage;
        a.stage = 0;
        a.Us = lv->U;
        a.U0 = lv->U;
        a.Uout = lv->U1;
        a.dt = scratch;
        a.cmax = reinterpret_cast<unsigned long long*>(scratch + 1);
        a.err = reinterpret_cast<unsigned int*>(scratch + 2);
        auto launch = [&](int sh, int od, int tm) {
            a.order = od;
            return launch_stage(&lv->p, a, st, 0, sh, tm ? &lv->maps[0] : nullptr);
        };
        const int rc = tune_candidates(launch, st, 2, &c, lv->maps[0].valid ? 2 : 1);
        cudaStreamSynchronize(st);
        cudaFree(scratch);
        if (rc) return rc;
        tune_store(key, c);
    }
    lv->shape = c.shape;
    lv->order = c.order;
    lv->use_tma = c.tma && lv->maps[0].valid;
    lv->tuned = true;
    return COMPAS_B200_OK;
}

// The launches of one coarse step: ComputeDt, then three (fill, stage) pairs, then t += dt.
static StepParams level_step_params(const compas_b200_level* lv) {
    StepParams sp;
    sp.cfl = lv->p.cfl;
    sp.dx[0] = lv->g.dx[0];
    sp.dx[1] = lv->g.dx[1];
    sp.dx[2] = lv->g.dx[2];
    sp.D = lv->p.dim;
    sp.limiter = lv->p.change_limiter;
    sp.dts = lv->dts;
    sp.dts_cap = lv->dts_cap;
    return sp;
}

static int enqueue_step(compas_b200_level* lv, cudaStream_t st) {
    const compas_b200_parm* p = &lv->p;
    const compas_b200_geom* g = &lv->g;
    const StepParams sp = level_step_params(lv);
    step_begin_kernel<<<1, 1, 0, st>>>(lv->ctl, sp);
    CUDA_TRY(cudaGetLastError());
    StageArgs a = base_args(p, g);
    a.mode = kModeStage;
    a.dt = &lv->ctl->dt;
    a.done = &lv->ctl->done;
    a.cmax = &lv->ctl->cmax;
    a.err = &lv->ctl->err;
    double* bufs_in[3] = {lv->U, lv->U1, lv->U2};
    double* bufs_out[3] = {lv->U1, lv->U2, lv->U};
    int rc;
    a.order = lv->order;
    for (int s = 0; s < 3; ++s) {
        if ((rc = launch_fill(p, g, bufs_in[s], st))) return rc;
        a.stage = s;
        a.Us = bufs_in[s];
        a.U0 = lv->U;
        a.Uout = bufs_out[s];
        if ((rc = launch_stage(p, a, st, 0, lv->shape, lv->use_tma ? &lv->maps[s] : nullptr))) return rc;
    }
    step_end_kernel<<<1, 1, 0, st>>>(lv->ctl);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

// ---- bound-preserving level advance (FiniteVolume.ID_Bound = 1) ----------------------------------
// The step of Evolve with its energy check (source/Class_Compressible_PhaseField.cpp:236-306) and the
// checks after every stage of ThirdOrderSSPRK (:4014-4030, :4049-4065, :4086-4102). A stage whose new
// state has a negative energy bound somewhere ends the step: its later launches do nothing, the host
// reads the three stages' bounds after the step, restores the state the step started from, computes
// the wave speeds of that state with the general bound (ID_Lambda = 0: CalculateInitialcmax under
// ID_Return = 1, :4481-4483), the step's dt again (ComputeDt, limited against the failed dt), and
// takes the step with ID_Lambda = 0. One host synchronisation per step, as the reference's host
// reductions after every stage need. If the step taken again still violates the bound, the level
// keeps the state it started from, sets COMPAS_B200_ERR_BOUND and stops (the reference goes on from
// the violating stage state).
__global__ void bp_restart_kernel(StepCtl* s, unsigned int err) {
    s->cmax = 0ull;  // RemakeAllLevelsFromData resets c_max
    s->err = err;    // the failed attempt's status bits are dropped with its state
}

__global__ void bp_fail_kernel(StepCtl* s) {
    s->err |= COMPAS_B200_ERR_BOUND;
    s->done = 1;
}

struct BpHostView {
    StepCtl ctl;
    unsigned long long eb[3];
};

static int bp_enqueue_stages(compas_b200_level* lv, int id_lambda, cudaStream_t st) {
    const compas_b200_parm* p = &lv->p;
    const compas_b200_geom* g = &lv->g;
    BpLevel* b = lv->bp;
    CUDA_TRY(cudaMemsetAsync(b->eb, 0xff, 3 * sizeof(unsigned long long), st));
    double* in[3] = {lv->U, lv->U1, lv->U2};
    double* out[3] = {lv->U1, lv->U2, lv->U};
    for (int s = 0; s < 3; ++s) {
        int rc;
        if ((rc = launch_fill(p, g, in[s], st))) return rc;
        if ((rc = bp_stage(p, g, b->faces, in[s], lv->U, out[s], kModeStage, s, &lv->ctl->dt, id_lambda,
                           &lv->ctl->done, b->eb, s, b->eb + s, &lv->ctl->cmax, &lv->ctl->err, st)))
            return rc;
    }
    lv->launches += 9;
    return COMPAS_B200_OK;
}

static int bp_read(compas_b200_level* lv, BpHostView* h, cudaStream_t st) {
    CUDA_TRY(cudaMemcpyAsync(&h->ctl, lv->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(h->eb, lv->bp->eb, sizeof(h->eb), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return COMPAS_B200_OK;
}

static bool bp_violated(const BpHostView& h) {
    for (int s = 0; s < 3; ++s)
        if (bp_key_negative(h.eb[s])) return true;
    return false;
}

static int bp_advance(compas_b200_level* lv, int nsteps, cudaStream_t st) {
    const compas_b200_parm* p = &lv->p;
    const compas_b200_geom* g = &lv->g;
    const StepParams sp = level_step_params(lv);
    BpHostView h;
    int rc;
    CUDA_TRY(cudaMemcpyAsync(&h.ctl, lv->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int s = 0; s < nsteps && !h.ctl.done; ++s) {
        const unsigned int err0 = h.ctl.err;
        step_begin_kernel<<<1, 1, 0, st>>>(lv->ctl, sp);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(lv->bp->Usave, lv->U, lv->bytes, cudaMemcpyDeviceToDevice, st));
        lv->launches += 1;
        if ((rc = bp_enqueue_stages(lv, 1, st))) return rc;
        if ((rc = bp_read(lv, &h, st))) return rc;
        if (h.ctl.done) break;
        if (bp_violated(h)) {
            ++lv->bp_restarts;
            CUDA_TRY(cudaMemcpyAsync(lv->U, lv->bp->Usave, lv->bytes, cudaMemcpyDeviceToDevice, st));
            bp_restart_kernel<<<1, 1, 0, st>>>(lv->ctl, err0);
            CUDA_TRY(cudaGetLastError());
            if ((rc = launch_fill(p, g, lv->U, st))) return rc;
            BpFaceArgs fa = bp_face_args(p, g, lv->U, 0);
            fa.cmax = &lv->ctl->cmax;
            fa.err = &lv->ctl->err;
            if ((rc = launch_bp_faces(fa, st))) return rc;
            step_begin_kernel<<<1, 1, 0, st>>>(lv->ctl, sp);
            CUDA_TRY(cudaGetLastError());
            lv->launches += 4;
            if ((rc = bp_enqueue_stages(lv, 0, st))) return rc;
            if ((rc = bp_read(lv, &h, st))) return rc;
            if (h.ctl.done) break;
            if (bp_violated(h)) {
                CUDA_TRY(cudaMemcpyAsync(lv->U, lv->bp->Usave, lv->bytes, cudaMemcpyDeviceToDevice, st));
                bp_fail_kernel<<<1, 1, 0, st>>>(lv->ctl);
                CUDA_TRY(cudaGetLastError());
                lv->launches += 1;
                break;
            }
        }
        step_end_kernel<<<1, 1, 0, st>>>(lv->ctl);
        CUDA_TRY(cudaGetLastError());
        lv->launches += 1;
        h.ctl.done = 0;
    }
    return COMPAS_B200_OK;
}

int compas_b200_level_advance(compas_b200_level* lv, int nsteps, double stop_time, int use_graph, void* stream) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    if (nsteps < 0) return fail(COMPAS_B200_EARG, "nsteps must be >= 0");
    cudaStream_t st = (cudaStream_t)stream;
    set_time_kernel<<<1, 1, 0, st>>>(lv->ctl, 0.0, stop_time, 0);
    CUDA_TRY(cudaGetLastError());
    lv->launches += 1;
    int rc;
    if (lv->need_init) {
        // CalculateInitialcmax (source/Class_Compressible_PhaseField.cpp:4501-4605)
        if ((rc = launch_fill(&lv->p, &lv->g, lv->U, st))) return rc;
        if (lv->bp) {
            // through the bound-preserving branch of the flux functor, ID_Lambda = 1
            BpFaceArgs fa = bp_face_args(&lv->p, &lv->g, lv->U, 1);
            fa.cmax = &lv->ctl->cmax;
            fa.err = &lv->ctl->err;
            if ((rc = launch_bp_faces(fa, st))) return rc;
        } else {
            StageArgs a = base_args(&lv->p, &lv->g);
            a.Us = lv->U;
            a.mode = kModeCmax;
            a.cmax = &lv->ctl->cmax;
            a.err = &lv->ctl->err;
            if ((rc = launch_stage(&lv->p, a, st))) return rc;
        }
        lv->launches += 2;
        lv->need_init = false;
    }
    if (nsteps == 0) return COMPAS_B200_OK;
    if (lv->bp) return bp_advance(lv, nsteps, st);
    if (lv->p.autotune && !lv->tuned && !lv->forced && !lv->p.thinc) {
        if ((rc = tune_level(lv, st))) return rc;
        if (lv->graph) {
            cudaGraphExecDestroy(lv->graph);
            lv->graph = nullptr;
        }
    }
    if (lv->pf) {
        // Evolve (source/Class_Compressible_PhaseField.cpp:171-330): each hyperbolic step is followed by
        // a Phase-Field step of the same dt; its host loop reads dt, max|u| and max|grad Q|.
        for (int s = 0; s < nsteps; ++s) {
            if ((rc = enqueue_step(lv, st))) return rc;
            lv->launches += 8;
            StepCtl h;
            CUDA_TRY(cudaMemcpyAsync(&h, lv->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            if (h.done || h.err) break;
            PfInfo info;
            std::string msg;
            if ((rc = pf_grad_q(lv->pf, &lv->p, lv->U, h.dt, st, &info, &msg))) return fail(rc, msg);
            lv->pf_last = info;
            const double* gq[3] = {pf_gq(lv->pf, 0), pf_gq(lv->pf, 1), lv->p.dim == 3 ? pf_gq(lv->pf, 2) : nullptr};
            int sub = 0;
            if ((rc = pf_advance(&lv->p, &lv->g, lv->U, lv->U1, lv->U2, gq, pf_dt_slot(lv->pf), h.dt, info.gmax,
                                 &lv->ctl->err, st, &sub, &lv->launches)))
                return rc;
            lv->pf_substeps += sub;
        }
        return COMPAS_B200_OK;
    }
    if (use_graph) {
        if (!lv->graph || lv->graph_stream != st) {
            if (lv->graph) {
                cudaGraphExecDestroy(lv->graph);
                lv->graph = nullptr;
            }
            // capture on a private stream so a legacy default stream can be used by the caller
            cudaStream_t cap;
            CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            cudaGraph_t graph;
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) {
                cudaStreamDestroy(cap);
                return fail(COMPAS_B200_ECUDA, std::string("begin capture: ") + cudaGetErrorString(e));
            }
            rc = enqueue_step(lv, cap);
            e = cudaStreamEndCapture(cap, &graph);
            cudaStreamDestroy(cap);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("end capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&lv->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("instantiate: ") + cudaGetErrorString(e));
            lv->graph_stream = st;
        }
        for (int s = 0; s < nsteps; ++s) CUDA_TRY(cudaGraphLaunch(lv->graph, st));
    } else {
        for (int s = 0; s < nsteps; ++s)
            if ((rc = enqueue_step(lv, st))) return rc;
    }
    lv->launches += 8LL * nsteps;
    return COMPAS_B200_OK;
}

// One step from a padded host state to a padded host state. The state moves in slabs of whole tile
// layers along the slowest direction (z in 3D, y in 2D): slab j is copied in on a copy stream while the
// stages of earlier slabs run, stage s of slab j runs once stage s-1 has written slabs j-1..j+1 (the
// stencil reaches 3 cells, a tile layer is 8 or 16), and slab j is copied out on a second copy stream
// as soon as the last stage has written it, so both copy directions overlap the stages. The kernels and
// tiles are those of compas_b200_level_advance (tile order 0), so the result is bit-identical to
// set_state + advance(1) + download. Falls back to that sequence for the first step of a level (the
// t = 0 wave-speed pass and the autotuner need the whole state), a periodic slab direction, a Phase-Field
// level or slabs < 2.
int compas_b200_level_step_host(compas_b200_level* lv, const double* host_in, double* host_out, int slabs,
                                void* stream) {
    if (!lv || !host_in || !host_out) return fail(COMPAS_B200_EARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const compas_b200_parm* p = &lv->p;
    const compas_b200_geom* g = &lv->g;
    const int D = p->dim, sd = D - 1;  // slab direction
    const int TS = (D == 2) ? kTile2 : kTile3;
    const int layers = (g->n[sd] + TS - 1) / TS;
    const int C = std::min(std::min(slabs, layers), 64);
    const bool tune_pending = p->autotune && !lv->tuned && !lv->forced && !p->thinc;
    if (lv->pf || lv->bp || lv->need_init || tune_pending || g->lo_bc[sd] == 0 || C < 2) {
        int rc;
        if ((rc = compas_b200_level_set_state(lv, host_in, 0, stream))) return rc;
        if ((rc = compas_b200_level_advance(lv, 1, 1.0e300, 1, stream))) return rc;
        return compas_b200_level_download(lv, host_out, 0, stream);
    }
    if (!lv->h2d) {
        CUDA_TRY(cudaStreamCreateWithFlags(&lv->h2d, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&lv->d2h, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&lv->ev_start, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&lv->ev_done, cudaEventDisableTiming));
        for (int c = 0; c < 64; ++c) {
            CUDA_TRY(cudaEventCreateWithFlags(&lv->ev_in[c], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&lv->ev_out[c], cudaEventDisableTiming));
        }
    }
    const Grid G = make_grid(p, g);
    const int gl = (D == 3) ? G.gz : G.ng;                 // ghost planes along the slab direction
    const long long unit = (D == 3) ? G.pxy : G.px;        // doubles per padded plane of one component
    const int N = nstate(p);
    const int layer_tiles = (D == 3) ? ((g->n[0] + TS - 1) / TS) * ((g->n[1] + TS - 1) / TS) : (g->n[0] + TS - 1) / TS;
    // slab c: tile layers [L0[c], L0[c+1]); valid planes [V0[c], V0[c+1]); padded planes [P0[c], P0[c+1])
    int L0[65], V0[65], P0[65];
    for (int c = 0; c <= C; ++c) {
        L0[c] = (int)((long long)c * layers / C);
        V0[c] = std::min(L0[c] * TS, g->n[sd]);
        P0[c] = (c == 0) ? 0 : (c == C ? g->n[sd] + 2 * gl : V0[c] + gl);
    }
    auto copy = [&](double* dst, const double* src, int c, cudaMemcpyKind kind, cudaStream_t s) {
        const size_t off = (size_t)P0[c] * unit;
        const size_t width = (size_t)(P0[c + 1] - P0[c]) * unit * sizeof(double);
        return cudaMemcpy2DAsync(dst + off, (size_t)G.S * sizeof(double), src + off, (size_t)G.S * sizeof(double), width,
                                 (size_t)N, kind, s);
    };
    // ghost planes filled with slab c: its own planes, and the domain's ghost planes at the two ends
    auto fill = [&](double* U, int c) {
        const int l0 = (c == 0) ? -gl : V0[c];
        const int l1 = (c == C - 1) ? g->n[sd] + gl : V0[c + 1];
        return launch_fill_slab(p, g, U, l0, l1, st);
    };
    set_time_kernel<<<1, 1, 0, st>>>(lv->ctl, 0.0, 1.0e300, 0);
    CUDA_TRY(cudaGetLastError());
    // the copies start after the caller's earlier work on its stream
    CUDA_TRY(cudaEventRecord(lv->ev_start, st));
    CUDA_TRY(cudaStreamWaitEvent(lv->h2d, lv->ev_start, 0));
    CUDA_TRY(cudaStreamWaitEvent(lv->d2h, lv->ev_start, 0));
    for (int c = 0; c < C; ++c) {
        CUDA_TRY(copy(lv->U, host_in, c, cudaMemcpyHostToDevice, lv->h2d));
        CUDA_TRY(cudaEventRecord(lv->ev_in[c], lv->h2d));
    }
    StepParams sp;
    sp.cfl = p->cfl;
    sp.dx[0] = g->dx[0];
    sp.dx[1] = g->dx[1];
    sp.dx[2] = g->dx[2];
    sp.D = D;
    sp.limiter = p->change_limiter;
    sp.dts = lv->dts;
    sp.dts_cap = lv->dts_cap;
    step_begin_kernel<<<1, 1, 0, st>>>(lv->ctl, sp);
    CUDA_TRY(cudaGetLastError());
    StageArgs a = base_args(p, g);
    a.mode = kModeStage;
    a.dt = &lv->ctl->dt;
    a.done = &lv->ctl->done;
    a.cmax = &lv->ctl->cmax;
    a.err = &lv->ctl->err;
    a.order = 0;
    double* bufs_in[3] = {lv->U, lv->U1, lv->U2};
    double* bufs_out[3] = {lv->U1, lv->U2, lv->U};
    int rc;
    for (int w = 0; w < C + 3; ++w) {
        if (w < C) {
            CUDA_TRY(cudaStreamWaitEvent(st, lv->ev_in[w], 0));
            if ((rc = fill(lv->U, w))) return rc;
        }
        for (int s = 0; s < 3; ++s) {
            const int c = w - 1 - s;
            if (c < 0 || c >= C) continue;
            a.stage = s;
            a.Us = bufs_in[s];
            a.U0 = lv->U;
            a.Uout = bufs_out[s];
            a.tile_base = L0[c] * layer_tiles;
            a.tile_count = (L0[c + 1] - L0[c]) * layer_tiles;
            if ((rc = launch_stage(p, a, st, 0, lv->shape, lv->use_tma ? &lv->maps[s] : nullptr))) return rc;
            if (s < 2) {
                if ((rc = fill(bufs_out[s], c))) return rc;
            } else {
                CUDA_TRY(cudaEventRecord(lv->ev_out[c], st));
                CUDA_TRY(cudaStreamWaitEvent(lv->d2h, lv->ev_out[c], 0));
                CUDA_TRY(copy(host_out, lv->U, c, cudaMemcpyDeviceToHost, lv->d2h));
            }
        }
    }
    step_end_kernel<<<1, 1, 0, st>>>(lv->ctl);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(lv->ev_done, lv->d2h));
    CUDA_TRY(cudaStreamWaitEvent(st, lv->ev_done, 0));
    lv->launches += 3 + 6LL * C;
    return COMPAS_B200_OK;
}

int compas_b200_level_kernel(const compas_b200_level* lv, int* shape, int* order) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    if (shape) *shape = lv->shape;
    if (order) *order = lv->order;
    return COMPAS_B200_OK;
}

int compas_b200_level_tma(const compas_b200_level* lv) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    return lv->use_tma ? 1 : 0;
}

int compas_b200_level_set_kernel(compas_b200_level* lv, int shape, int order) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    if (shape < 0 || shape >= kShapes || order < 0 || order >= kOrders)
        return fail(COMPAS_B200_EARG, "shape in [0, " + std::to_string(kShapes) + "), order in [0, " +
                                          std::to_string(kOrders) + ")");
    lv->shape = shape;
    lv->order = order;
    lv->forced = true;
    if (lv->graph) {
        cudaGraphExecDestroy(lv->graph);
        lv->graph = nullptr;
    }
    return COMPAS_B200_OK;
}

long long compas_b200_level_bound_restarts(const compas_b200_level* lv) { return lv ? lv->bp_restarts : 0; }

int compas_b200_energy_bound_min(const compas_b200_parm* p, const compas_b200_geom* g, const double* U,
                                 double* min_dev, void* stream) {
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U || !min_dev) return fail(COMPAS_B200_EARG, "null argument");
    if (p->physics == COMPAS_B200_SIXEQS || p->physics == COMPAS_B200_SIXEQS_IE_NPHASE)
        return fail(COMPAS_B200_EUNSUPPORTED, "the energy bound is this engine's for FIVEEQS and FIVEEQS_NPHASE");
    cudaStream_t st = (cudaStream_t)stream;
    const Grid G = make_grid(p, g);
    const long long cells = (long long)G.n[0] * G.n[1] * (p->dim == 3 ? G.n[2] : 1);
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((cells + 127) / 128, 148LL * 16));
    // the result slot holds the ordered key of the running minimum, then the value
    auto* key = reinterpret_cast<unsigned long long*>(min_dev);
    CUDA_TRY(cudaMemsetAsync(key, 0xff, sizeof(unsigned long long), st));
    CUDA_TRY(launch_bp_min_model(U, G, make_eos(p), p->dim, p->physics, p->nphase, key, blocks, st));
    bp_key_to_double_kernel<<<1, 1, 0, st>>>(key, min_dev);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

int compas_b200_level_sync(compas_b200_level* lv, double* t, int* steps, unsigned int* status) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    StepCtl h;
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(&h, lv->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost));
    if (t) *t = h.t;
    if (steps) *steps = h.steps;
    if (status) *status = h.err;
    const unsigned int fatal = COMPAS_B200_ERR_NAN | COMPAS_B200_ERR_COVOLUME | COMPAS_B200_ERR_CFL;
    if (h.err & fatal) return fail(COMPAS_B200_ESTATE, "status word " + std::to_string(h.err));
    return COMPAS_B200_OK;
}

int compas_b200_level_dts(compas_b200_level* lv, double* dts, int n) {
    if (!lv || !dts) return fail(COMPAS_B200_EARG, "null argument");
    if (n > lv->dts_cap) n = lv->dts_cap;
    if (n <= 0) return COMPAS_B200_OK;
    CUDA_TRY(cudaMemcpy(dts, lv->dts, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return COMPAS_B200_OK;
}


// ---- batched independent cases (box list) ------------------------------------------------------

static int batch_sync_list(compas_b200_batch* b, cudaStream_t st) {
    const int nb = (int)b->cases.size();
    std::vector<BoxDesc> boxes(nb);
    std::vector<int> tile_off(nb + 1, 0), slots(nb, 0);
    std::vector<long long> ghost_off(nb + 1, 0);
    for (int i = 0; i < nb; ++i) {
        const BatchCase& c = b->cases[i];
        BoxDesc& B = boxes[i];
        std::memset(&B, 0, sizeof(B));
        B.g = make_grid(&c.p, &c.g);
        B.e = make_eos(&c.p);
        for (int k = 0; k < 3; ++k) B.U[k] = c.U[k];
        StepCtl* ctl = b->d_ctl + c.slot;
        B.dt = &ctl->dt;
        B.done = &ctl->done;
        B.cmax = &ctl->cmax;
        B.err = &ctl->err;
        for (int d = 0; d < 3; ++d) {
            B.lo_bc[d] = c.g.lo_bc[d];
            B.hi_bc[d] = c.g.hi_bc[d];
        }
        B.id_k = c.p.source_term;
        B.relax = (c.p.physics == COMPAS_B200_SIXEQS || c.p.physics == COMPAS_B200_SIXEQS_IE_NPHASE) ? c.p.relaxation : 0;
        B.riemann = c.p.id_riemann;
        B.muscl = c.p.id_weno ? (c.p.id_limiter == 3 ? 10 : (c.p.id_limiter == 4 ? 11 : -1)) : c.p.id_limiter;
        B.trace = c.p.relax_trace;
        B.tiles = tile_count(b->dim, B.g);
        B.ghosts = ghost_count(B.g);
        tile_off[i + 1] = tile_off[i] + B.tiles;
        ghost_off[i + 1] = ghost_off[i] + B.ghosts;
        slots[i] = c.slot;
    }
    if (nb > 0) {
        CUDA_TRY(cudaMemcpyAsync(b->d_boxes, boxes.data(), sizeof(BoxDesc) * nb, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(b->d_slots, slots.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemcpyAsync(b->d_tile_off, tile_off.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(b->d_ghost_off, ghost_off.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(b->d_nbox, &nb, sizeof(int), cudaMemcpyHostToDevice, st));
    // pageable sources: make the copies complete before the vectors go out of scope
    CUDA_TRY(cudaStreamSynchronize(st));
    return COMPAS_B200_OK;
}

int compas_b200_batch_create(int physics, int dim, int id_limiter, int precision, int capacity,
                             compas_b200_batch** out) {
    return compas_b200_batch_create_nphase(physics, dim, 2, id_limiter, precision, capacity, out);
}

int compas_b200_batch_create_nphase(int physics, int dim, int nphase, int id_limiter, int precision, int capacity,
                                    compas_b200_batch** out) {
    if (!out) return fail(COMPAS_B200_EARG, "null output");
    *out = nullptr;
    compas_b200_parm probe;
    int rc = compas_b200_parm_init_nphase(&probe, physics, dim, nphase);
    if (rc) return rc;
    if (physics == COMPAS_B200_FIVEEQS_NPHASE && !nphase_built(dim, nphase))
        return fail(COMPAS_B200_EUNSUPPORTED, "FIVEEQS_NPHASE batches: NPHASE 2, 3, 4 in 2D and 3 in 3D");
    if (physics == COMPAS_B200_SIXEQS_IE_NPHASE && !sixn_built(dim, nphase))
        return fail(COMPAS_B200_EUNSUPPORTED, "SIXEQS_IE_NPHASE batches: NPHASE 2, 3 in 2D and 3 in 3D");
    if (id_limiter != 5 && id_limiter != 6) return fail(COMPAS_B200_EUNSUPPORTED, "WENO5 (5) or WENO5B (6)");
    if (precision != 0 && precision != 1) return fail(COMPAS_B200_EARG, "precision 0 or 1");
    if (capacity < 1 || capacity > (1 << 20)) return fail(COMPAS_B200_EARG, "capacity out of range");
    auto* b = new compas_b200_batch();
    b->physics = physics;
    b->dim = dim;
    b->nphase = nphase;
    b->limiter = id_limiter;
    b->precision = precision;
    b->capacity = capacity;
    for (int i = capacity - 1; i >= 0; --i) b->free_slots.push_back(i);
    cudaError_t e = cudaMalloc(&b->d_boxes, sizeof(BoxDesc) * capacity);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_nbox, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tile_off, sizeof(int) * (capacity + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ghost_off, sizeof(long long) * (capacity + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_slots, sizeof(int) * capacity);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ctl, sizeof(StepCtl) * capacity);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_cs, sizeof(CaseStep) * capacity);
    if (e == cudaSuccess) e = cudaMemset(b->d_ctl, 0, sizeof(StepCtl) * capacity);
    if (e == cudaSuccess) e = cudaMemset(b->d_nbox, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_tile_off, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_ghost_off, 0, sizeof(long long));
    if (e != cudaSuccess) {
        compas_b200_batch_destroy(b);
        cudaGetLastError();
        return fail(COMPAS_B200_ENOMEM, std::string("batch allocation: ") + cudaGetErrorString(e));
    }
    *out = b;
    return COMPAS_B200_OK;
}

int compas_b200_batch_destroy(compas_b200_batch* b) {
    if (!b) return COMPAS_B200_OK;
    cudaDeviceSynchronize();
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& c : b->cases)
        for (int k = 0; k < 3; ++k) cudaFree(c.U[k]);
    cudaFree(b->d_boxes);
    cudaFree(b->d_nbox);
    cudaFree(b->d_tile_off);
    cudaFree(b->d_ghost_off);
    cudaFree(b->d_slots);
    cudaFree(b->d_ctl);
    cudaFree(b->d_cs);
    delete b;
    return COMPAS_B200_OK;
}

int compas_b200_batch_add(compas_b200_batch* b, const compas_b200_parm* p, const compas_b200_geom* g,
                          const double* U, int is_device, double stop_time, int max_steps, void* stream,
                          int* case_id) {
    if (!b || !U) return fail(COMPAS_B200_EARG, "null argument");
    int rc = check_args(p, g);
    if (rc) return rc;
    if (p->physics != b->physics || p->dim != b->dim || p->id_limiter != b->limiter || p->precision != b->precision ||
        (nphase_model(p->physics) && p->nphase != b->nphase))
        return fail(COMPAS_B200_EARG, "a batch holds cases of one model, dimension, number of phases, scheme and precision");
    if (p->thinc) return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.THINC = 1 runs on the level API, not in a batch");
    if (p->id_bound) return fail(COMPAS_B200_EUNSUPPORTED, "FiniteVolume.ID_Bound = 1 runs on the level API, not in a batch");
    if (b->free_slots.empty()) return fail(COMPAS_B200_ENOMEM, "batch capacity reached");
    if (max_steps < 0) return fail(COMPAS_B200_EARG, "max_steps must be >= 0");
    cudaStream_t st = (cudaStream_t)stream;
    BatchCase c;
    c.p = *p;
    c.g = *g;
    if (p->dim == 2) c.g.n[2] = 1;
    c.bytes = compas_b200_state_bytes(p, g);
    for (int k = 0; k < 3; ++k) {
        cudaError_t e = cudaMalloc(&c.U[k], c.bytes);
        if (e != cudaSuccess) {
            for (int j = 0; j < k; ++j) cudaFree(c.U[j]);
            cudaGetLastError();
            return fail(COMPAS_B200_ENOMEM, std::string("case allocation: ") + cudaGetErrorString(e));
        }
    }
    CUDA_TRY(cudaMemcpyAsync(c.U[0], U, c.bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    c.slot = b->free_slots.back();
    b->free_slots.pop_back();
    c.id = b->next_id++;
    StepCtl h;
    std::memset(&h, 0, sizeof(h));
    h.dt_prev = 1.e100;
    h.stop_time = stop_time;
    CaseStep cs;
    cs.cfl = p->cfl;
    cs.dx[0] = g->dx[0];
    cs.dx[1] = g->dx[1];
    cs.dx[2] = g->dx[2];
    cs.D = p->dim;
    cs.limiter = p->change_limiter;
    cs.max_steps = max_steps;
    cs.stop_time = stop_time;
    CUDA_TRY(cudaMemcpyAsync(b->d_ctl + c.slot, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(b->d_cs + c.slot, &cs, sizeof(cs), cudaMemcpyHostToDevice, st));
    // CalculateInitialcmax of the new case
    if ((rc = launch_fill(&c.p, &c.g, c.U[0], st))) return rc;
    StageArgs a = base_args(&c.p, &c.g);
    a.Us = c.U[0];
    a.mode = kModeCmax;
    a.cmax = &(b->d_ctl + c.slot)->cmax;
    a.err = &(b->d_ctl + c.slot)->err;
    if ((rc = launch_stage(&c.p, a, st))) return rc;
    b->launches += 2;
    b->cases.push_back(c);
    b->bytes_in_use += 3 * c.bytes;
    if (case_id) *case_id = c.id;
    return batch_sync_list(b, st);
}

int compas_b200_batch_remove(compas_b200_batch* b, int case_id, void* stream) {
    if (!b) return fail(COMPAS_B200_EARG, "null batch");
    cudaStream_t st = (cudaStream_t)stream;
    for (size_t i = 0; i < b->cases.size(); ++i) {
        if (b->cases[i].id != case_id) continue;
        BatchCase c = b->cases[i];
        b->cases.erase(b->cases.begin() + i);
        int rc = batch_sync_list(b, st);
        CUDA_TRY(cudaStreamSynchronize(st));
        for (int k = 0; k < 3; ++k) cudaFree(c.U[k]);
        b->free_slots.push_back(c.slot);
        b->bytes_in_use -= 3 * c.bytes;
        return rc;
    }
    return fail(COMPAS_B200_EARG, "no case with id " + std::to_string(case_id));
}

// Autotune the batch's box-list kernel on the cases admitted so far (all at t = 0 when the batch first
// advances): a stage-0 launch per candidate with each case's dt still 0, into each case's stage
// buffer; the wave speeds it adds equal the t = 0 pass's, so the step control is unchanged.
static int tune_batch(compas_b200_batch* b, cudaStream_t st) {
    long long tiles = 0;
    for (auto& c : b->cases) tiles += tile_count(b->dim, make_grid(&c.p, &c.g));
    long long tb = 1, nb = 1;
    while (tb < tiles) tb <<= 1;
    while (nb < (long long)b->cases.size()) nb <<= 1;
    const std::string key = tune_key(&b->cases[0].p, "list", tb, nb, 0);
    TuneChoice c;
    if (!tune_lookup(key, &c)) {
        auto launch = [&](int sh, int od, int) {
            ListArgs L{b->d_boxes, b->d_nbox, b->d_tile_off, kModeStage, 0, od};
            return launch_list(b->physics, b->dim, b->nphase, b->limiter, b->precision, L, st, sh);
        };
        int rc = tune_candidates(launch, st, 2, &c);
        if (rc) return rc;
        tune_store(key, c);
    }
    b->shape = c.shape;
    b->order = c.order;
    b->tuned = true;
    return COMPAS_B200_OK;
}

static int batch_enqueue_step(compas_b200_batch* b, cudaStream_t st) {
    step_begin_list_kernel<<<4, 256, 0, st>>>(b->d_ctl, b->d_cs, b->d_slots, b->d_nbox);
    CUDA_TRY(cudaGetLastError());
    const int N = nstate_of(b->physics, b->dim, b->nphase);
    int rc;
    for (int s = 0; s < 3; ++s) {
        FillListArgs F{b->d_boxes, b->d_nbox, b->d_ghost_off, N, b->dim, mom0_of(b->physics, b->nphase), s};
        fill_list_kernel<<<148 * 8, 256, 0, st>>>(F);
        CUDA_TRY(cudaGetLastError());
        ListArgs L{b->d_boxes, b->d_nbox, b->d_tile_off, kModeStage, s, b->order};
        if ((rc = launch_list(b->physics, b->dim, b->nphase, b->limiter, b->precision, L, st, b->shape))) return rc;
    }
    step_end_list_kernel<<<4, 256, 0, st>>>(b->d_ctl, b->d_slots, b->d_nbox);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

int compas_b200_batch_advance(compas_b200_batch* b, int nsteps, int use_graph, void* stream) {
    if (!b) return fail(COMPAS_B200_EARG, "null batch");
    if (nsteps < 0) return fail(COMPAS_B200_EARG, "nsteps must be >= 0");
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (!b->tuned && !b->forced && !b->cases.empty() && b->cases[0].p.autotune && nsteps > 0) {
        if ((rc = tune_batch(b, st))) return rc;
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
    }
    if (use_graph) {
        if (!b->graph || b->graph_stream != st) {
            if (b->graph) {
                cudaGraphExecDestroy(b->graph);
                b->graph = nullptr;
            }
            cudaStream_t cap;
            CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            cudaGraph_t graph;
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) {
                cudaStreamDestroy(cap);
                return fail(COMPAS_B200_ECUDA, std::string("begin capture: ") + cudaGetErrorString(e));
            }
            rc = batch_enqueue_step(b, cap);
            e = cudaStreamEndCapture(cap, &graph);
            cudaStreamDestroy(cap);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("end capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&b->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(COMPAS_B200_ECUDA, std::string("instantiate: ") + cudaGetErrorString(e));
            b->graph_stream = st;
        }
        for (int s = 0; s < nsteps; ++s) CUDA_TRY(cudaGraphLaunch(b->graph, st));
    } else {
        for (int s = 0; s < nsteps; ++s)
            if ((rc = batch_enqueue_step(b, st))) return rc;
    }
    b->launches += 8LL * nsteps;
    return COMPAS_B200_OK;
}

int compas_b200_batch_kernel(const compas_b200_batch* b, int* shape, int* order) {
    if (!b) return fail(COMPAS_B200_EARG, "null batch");
    if (shape) *shape = b->shape;
    if (order) *order = b->order;
    return COMPAS_B200_OK;
}

int compas_b200_batch_set_kernel(compas_b200_batch* b, int shape, int order) {
    if (!b) return fail(COMPAS_B200_EARG, "null batch");
    if (shape < 0 || shape >= kShapes || order < 0 || order >= kOrders)
        return fail(COMPAS_B200_EARG, "shape in [0, " + std::to_string(kShapes) + "), order in [0, " +
                                          std::to_string(kOrders) + ")");
    b->shape = shape;
    b->order = order;
    b->forced = true;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return COMPAS_B200_OK;
}

int compas_b200_batch_poll(compas_b200_batch* b, int* ids, double* t, int* steps, int* done, unsigned int* status,
                           int cap) {
    if (!b) return fail(COMPAS_B200_EARG, "null batch");
    CUDA_TRY(cudaDeviceSynchronize());
    std::vector<StepCtl> h(b->capacity);
    CUDA_TRY(cudaMemcpy(h.data(), b->d_ctl, sizeof(StepCtl) * b->capacity, cudaMemcpyDeviceToHost));
    const int n = std::min<int>(cap, (int)b->cases.size());
    for (int i = 0; i < n; ++i) {
        const BatchCase& c = b->cases[i];
        const StepCtl& s = h[c.slot];
        if (ids) ids[i] = c.id;
        if (t) t[i] = s.t;
        if (steps) steps[i] = s.steps;
        if (done) done[i] = s.done;
        if (status) status[i] = s.err;
    }
    return (int)b->cases.size();
}

int compas_b200_batch_download(compas_b200_batch* b, int case_id, double* dst, int is_device, void* stream) {
    if (!b || !dst) return fail(COMPAS_B200_EARG, "null argument");
    for (const auto& c : b->cases)
        if (c.id == case_id) {
            CUDA_TRY(cudaMemcpyAsync(dst, c.U[0], c.bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                     (cudaStream_t)stream));
            return COMPAS_B200_OK;
        }
    return fail(COMPAS_B200_EARG, "no case with id " + std::to_string(case_id));
}

long long compas_b200_batch_bytes(compas_b200_batch* b) { return b ? b->bytes_in_use : 0; }

long long compas_b200_batch_launches(compas_b200_batch* b) { return b ? b->launches : 0; }

}  // extern "C"

#include "amr_api.inc"

int compas_b200_tag_cells(const compas_b200_parm* p, const compas_b200_geom* g, const double* U,
                          const compas_b200_tag_criterion* criteria, int ncriteria, unsigned char* tags,
                          void* stream) {
    using namespace compas;
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U || !tags) return fail(COMPAS_B200_EARG, "null state or tag array");
    if (ncriteria < 0 || ncriteria > kMaxTagCriteria || (ncriteria > 0 && !criteria))
        return fail(COMPAS_B200_EARG, "between 0 and " + std::to_string(kMaxTagCriteria) + " tagging criteria");
    if (nphase_model(p->physics))
        return fail(COMPAS_B200_EUNSUPPORTED, "refinement tagging: FIVEEQS and SIXEQS");
    if (g->ng < 2) return fail(COMPAS_B200_EARG, "refinement tagging needs two ghost cells");
    const int nderived = (p->physics == COMPAS_B200_SIXEQS) ? 21 : 18;
    TagArgs a;
    std::memset(&a, 0, sizeof(a));
    a.U = U;
    a.g = make_grid(p, g);
    a.e = make_eos(p);
    a.cv1 = p->cv_1;
    a.cv2 = p->cv_2;
    a.ncrit = ncriteria;
    a.tags = tags;
    for (int v = 0; v < ncriteria; ++v) {
        const compas_b200_tag_criterion& c = criteria[v];
        if (c.kind < COMPAS_B200_TAG_GRAD || c.kind > COMPAS_B200_TAG_RANGE)
            return fail(COMPAS_B200_EARG, "tagging criterion kind must be GRAD, LESS, GREATER or RANGE");
        if (c.var < 0 || c.var >= (c.derived ? nderived : nstate(p)))
            return fail(COMPAS_B200_EARG, "tagging criterion variable out of range");
        a.c[v].var = c.var;
        a.c[v].derived = c.derived ? 1 : 0;
        a.c[v].kind = c.kind;
        a.c[v].v0 = c.v0;
        a.c[v].v1 = c.v1;
    }
    const long long n = (long long)a.g.n[0] * a.g.n[1] * a.g.n[2];
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32));
    cudaStream_t st = (cudaStream_t)stream;
    if (p->physics == COMPAS_B200_SIXEQS) {
        if (p->dim == 2) tag_kernel<SixEq<2>><<<blocks, 256, 0, st>>>(a);
        else tag_kernel<SixEq<3>><<<blocks, 256, 0, st>>>(a);
    } else {
        if (p->dim == 2) tag_kernel<FiveEq<2>><<<blocks, 256, 0, st>>>(a);
        else tag_kernel<FiveEq<3>><<<blocks, 256, 0, st>>>(a);
    }
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

int compas_b200_derive(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, const int* vars,
                       const int* derived, int nvars, double* out, void* stream) {
    using namespace compas;
    int rc = check_args(p, g);
    if (rc) return rc;
    if (!U || !out || (nvars > 0 && (!vars || !derived))) return fail(COMPAS_B200_EARG, "null argument");
    if (nvars < 0 || nvars > kMaxDerive) return fail(COMPAS_B200_EARG, "between 0 and 32 variables");
    if (nphase_model(p->physics))
        return fail(COMPAS_B200_EUNSUPPORTED, "derived variables: FIVEEQS and SIXEQS");
    if (g->ng < 2) return fail(COMPAS_B200_EARG, "derived variables need two ghost cells");
    const int nderived = (p->physics == COMPAS_B200_SIXEQS) ? 21 : 18;
    DeriveArgs a;
    std::memset(&a, 0, sizeof(a));
    a.t.U = U;
    a.t.g = make_grid(p, g);
    a.t.e = make_eos(p);
    a.t.cv1 = p->cv_1;
    a.t.cv2 = p->cv_2;
    a.nv = nvars;
    a.out = out;
    for (int v = 0; v < nvars; ++v) {
        if (vars[v] < 0 || vars[v] >= (derived[v] ? nderived : nstate(p)))
            return fail(COMPAS_B200_EARG, "derived variable index out of range");
        a.var[v] = vars[v];
        a.derived[v] = derived[v] ? 1 : 0;
    }
    const long long n = (long long)a.t.g.n[0] * a.t.g.n[1] * a.t.g.n[2];
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32));
    cudaStream_t st = (cudaStream_t)stream;
    if (p->physics == COMPAS_B200_SIXEQS) {
        if (p->dim == 2) derive_kernel<SixEq<2>><<<blocks, 256, 0, st>>>(a);
        else derive_kernel<SixEq<3>><<<blocks, 256, 0, st>>>(a);
    } else {
        if (p->dim == 2) derive_kernel<FiveEq<2>><<<blocks, 256, 0, st>>>(a);
        else derive_kernel<FiveEq<3>><<<blocks, 256, 0, st>>>(a);
    }
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}

// ---- step control of a level, for checkpoint and restart ----------------------------------------
__global__ void set_control_kernel(StepCtl* s, double t, double dt_prev, unsigned long long cmax, int steps) {
    s->t = t;
    s->dt = 0.0;
    s->dt_prev = dt_prev;
    s->cmax = cmax;
    s->steps = steps;
    s->err = 0u;
    s->done = 0;
}

int compas_b200_level_get_control(compas_b200_level* lv, double* t, double* dt_prev, double* cmax, int* steps) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    CUDA_TRY(cudaDeviceSynchronize());
    StepCtl h;
    CUDA_TRY(cudaMemcpy(&h, lv->ctl, sizeof(h), cudaMemcpyDeviceToHost));
    if (t) *t = h.t;
    if (dt_prev) *dt_prev = h.dt_prev;
    if (cmax) std::memcpy(cmax, &h.cmax, sizeof(double));
    if (steps) *steps = h.steps;
    return COMPAS_B200_OK;
}

int compas_b200_level_set_control(compas_b200_level* lv, double t, double dt_prev, double cmax, int steps,
                                  void* stream) {
    if (!lv) return fail(COMPAS_B200_EARG, "null level");
    if (!(cmax >= 0.0) || steps < 0) return fail(COMPAS_B200_EARG, "cmax must be >= 0 and steps >= 0");
    unsigned long long bits;
    std::memcpy(&bits, &cmax, sizeof(bits));
    set_control_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(lv->ctl, t, dt_prev, bits, steps);
    CUDA_TRY(cudaGetLastError());
    lv->need_init = false;  // the next step's dt comes from the restored c_max, as in the run checkpointed
    return COMPAS_B200_OK;
}

// ---- THINC face values, for the per-face comparison with the reference's host function -------------
namespace compas {
__global__ void thinc_face_kernel(const double* beta, const double* sigma, const double* abar, const int* side,
                                  long long n, double* out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = thinc_alpha_face(beta[t], sigma[t], abar[t], side[t]);
}
}  // namespace compas

int compas_b200_thinc_face_values(const double* beta, const double* sigma, const double* abar, const int* side,
                                  long long n, double* out, void* stream) {
    using namespace compas;
    if (n < 0 || (n > 0 && (!beta || !sigma || !abar || !side || !out))) return fail(COMPAS_B200_EARG, "null argument");
    if (n == 0) return COMPAS_B200_OK;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 32);
    thinc_face_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(beta, sigma, abar, side, n, out);
    CUDA_TRY(cudaGetLastError());
    return COMPAS_B200_OK;
}
