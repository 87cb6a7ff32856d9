// Multi-level (AMR) advance of a fixed box hierarchy on the device: refinement ratio 2, subcycling,
// TVD-RK3 per level through the persistent box-list stage kernel, coarse-fine ghost cells by linear
// time interpolation and cell-conservative linear interpolation, conservative refluxing (with the
// five-equation non-conservative alpha1 source) and average-down.
//
// Reference orchestration (source/): timeStepWithSubcycling Class_Compressible_PhaseField.cpp:4359-4451,
// ThirdOrderSSPRK with flux registers :3937-4107 and :3472-3537, ComputeDt COMPAS.cpp:2249-2303,
// FillPatch / FillPatchStage COMPAS.cpp:1598-1799 with GetData :1953-1985, AverageDownTo :1549-1558,
// RefluxLev Class_Compressible5Eq_PhaseField.cpp:77-160. The AMReX operations (FillPatchTwoLevels,
// lincc_interp, FluxRegister, average_down) follow their documented semantics; lincc_interp is AMReX's
// CellConservativeLinear with linear limiting: per direction the central slopes of all components
// scaled by one factor shared by the components, the smallest ratio of a component's
// monotonized-central slope to its central slope (fine value u_c + sum_d off_d slope_d, off_d = -1/4 or
// +1/4).
//
// Layout: every box keeps four padded arrays (two alternating time levels, two stage states); the
// host builds, once per hierarchy, the tables of where every ghost cell, coarse-fine face and
// covered coarse cell takes its data from, so a level fill is three table-driven launches.
#pragma once

#include <vector>

namespace compas {

// ghost cell copied from a valid cell of a box of the same level (periodic images included)
struct AmrSame {
    int db, sb;
    long long dq, sq;
};
// ghost cell interpolated from the coarse level: stencil cells C, C-e0, C+e0, C-e1, C+e1 (, C-e2, C+e2)
// with, per stencil cell, the coarse box, the padded index and the components whose value changes
// sign through a reflecting boundary
struct AmrInterp {
    int db;
    long long dq;
    int cb[7];
    long long cq[7];
    unsigned odd[7];
    int par;  // bit d set: the fine cell is the upper child along d (offset +1/4)
};
// ghost cell outside the domain along one direction: mirror / extrapolation within the same box
struct AmrBc {
    int b;
    long long dq, sq;
    unsigned odd;
};
// coarse-fine face between an uncovered coarse cell and the fine region
struct AmrCf {
    int cbox;                  // coarse box of the uncovered coarse cell
    long long cq;              // its padded index
    int cface[3];              // face index in the coarse box (local, nodal along d)
    int d, hi_side;
    int fbox[4];               // fine boxes and local face indices of the 2^(D-1) fine faces
    int fface[4][3];
};
// covered coarse cell and its 2^D fine children
struct AmrAvg {
    int cb;
    long long cq;
    int fb[8];
    long long fq[8];
};

struct AmrBoxH {
    int lev;
    int lo[3], hi[3], n[3];
    Grid g;
    double* buf[4] = {nullptr, nullptr, nullptr, nullptr};  // time levels 0/1, stage states 1/2
    long long S;
};

struct AmrLevelH {
    std::vector<int> boxes;
    int dom[3];
    double dx[3];
    int parity = 0;  // buf[parity] is U_new, buf[1-parity] U_old
    double t_old = 0.0, t_new = 0.0, dt = 1.e100;
    double cmax = 0.0;
    // box-list launch of the level: descriptors for both parities
    BoxDesc* d_desc[2] = {nullptr, nullptr};
    int* d_nbox = nullptr;
    int* d_tile_off = nullptr;
    // step control of the level on the device
    double* d_dt = nullptr;
    unsigned long long* d_cmax = nullptr;
    int* d_done = nullptr;
    // tables
    AmrSame* d_same = nullptr;
    long long n_same = 0;
    AmrInterp* d_interp = nullptr;
    long long n_interp = 0;
    AmrBc* d_bc[3] = {nullptr, nullptr, nullptr};
    long long n_bc[3] = {0, 0, 0};
    // as the fine level of the pair (l-1, l): coarse-fine faces, registers, reflux groups
    AmrCf* d_cf = nullptr;
    int n_cf = 0;
    double* d_reg = nullptr;
    double* d_reg_nc = nullptr;
    int* d_groups = nullptr;  // start of each coarse-cell group in the face list, n_groups + 1 entries
    int n_groups = 0;
    AmrAvg* d_avg = nullptr;  // covered cells of level l-1
    long long n_avg = 0;
};

// ---- kernels -------------------------------------------------------------------------------------------
struct AmrBufs {
    double* const* p;          // p[box * 4 + k]
    const long long* S;        // component stride of each box
};

__global__ void amr_same_kernel(const AmrSame* t, long long n, AmrBufs B, int dk, int sk, int N) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const AmrSame e = t[q];
        double* dst = B.p[e.db * 4 + dk];
        const double* src = B.p[e.sb * 4 + sk];
        const long long Sd = B.S[e.db], Ss = B.S[e.sb];
        for (int c = 0; c < N; ++c) dst[c * Sd + e.dq] = src[c * Ss + e.sq];
    }
}

// mode 0: coarse new data, 1: coarse old data, 2: alpha old + beta new
__device__ __forceinline__ double amr_coarse(const AmrBufs& B, int cb, long long cq, int c, int knew, int kold, int mode,
                                             double alpha, double beta) {
    const long long S = B.S[cb];
    if (mode == 0) return B.p[cb * 4 + knew][c * S + cq];
    if (mode == 1) return B.p[cb * 4 + kold][c * S + cq];
    return alpha * B.p[cb * 4 + kold][c * S + cq] + beta * B.p[cb * 4 + knew][c * S + cq];
}

// pc: amr.Interpolater = pc_interp (the parent's value, AMReX PCInterp); else lincc_interp as restated in the
// file header: per direction the central slopes of all components, one monotonized-central factor shared
// by the components, u_f = u_c + sum_d +-1/4 slope_d
__global__ void amr_interp_kernel(const AmrInterp* t, long long n, AmrBufs B, int dk, int knew, int kold, int mode,
                                  double alpha, double beta, int N, int D, int pc) {
    constexpr int NMAX = 2 * COMPAS_B200_MAX_PHASES + 4;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const AmrInterp& e = t[q];
        double* dst = B.p[e.db * 4 + dk];
        const long long Sd = B.S[e.db];
        auto val = [&](int s, int c) {
            const double v = amr_coarse(B, e.cb[s], e.cq[s], c, knew, kold, mode, alpha, beta);
            return ((e.odd[s] >> c) & 1u) ? -1.0 * v : 1.0 * v;
        };
        double u[NMAX];
        for (int c = 0; c < N; ++c) u[c] = val(0, c);
        for (int d = 0; d < (pc ? 0 : D); ++d) {
            double dcs[NMAX];
            double sf = 1.0;
            for (int c = 0; c < N; ++c) {
                const double uc = val(0, c);
                const double um = val(1 + 2 * d, c), up = val(2 + 2 * d, c);
                const double dc = 0.5 * (up - um), df = 2.0 * (up - uc), db = 2.0 * (uc - um);
                double sx = (df * db >= 0.0) ? dmin(fabs(df), fabs(db)) : 0.0;
                sx = copysign(1.0, dc) * dmin(sx, fabs(dc));
                if (dc != 0.0) sf = dmin(sf, sx / dc);
                dcs[c] = dc;
            }
            const double off = ((e.par >> d) & 1) ? 0.25 : -0.25;
            for (int c = 0; c < N; ++c) u[c] = u[c] + off * (dcs[c] * sf);
        }
        for (int c = 0; c < N; ++c) dst[c * Sd + e.dq] = u[c];
    }
}

__global__ void amr_bc_kernel(const AmrBc* t, long long n, AmrBufs B, int k, int N) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const AmrBc e = t[q];
        double* a = B.p[e.b * 4 + k];
        const long long S = B.S[e.b];
        for (int c = 0; c < N; ++c) {
            const double v = a[c * S + e.sq];
            a[c * S + e.dq] = ((e.odd >> c) & 1u) ? -1.0 * v : 1.0 * v;
        }
    }
}

// face flux of face (i,j,k) (between cells i-1 and i along d) of a box with ghost-filled data U,
// by the same sequence of device functions as the stage kernel (stage_kernel.cuh, step 2b): WENO5 /
// WENO5B (SCHEME 5 / 6) or the three-cell schemes (SCHEME 2, `code` as StageArgs::muscl), the N-phase
// consistent limiter, the Riemann solver `id_riemann`
template <class M, int SCHEME, bool MIX>
__device__ void amr_face_flux(const double* U, const Grid& g, int d, int i, int j, int k, const Eos& e, int id_k,
                              int code, int id_riemann, double dxd, double* F, double* fnc, unsigned int* err) {
    using PT = typename std::conditional<MIX, float, double>::type;
    constexpr int N = M::N, D = M::D;
    constexpr bool NPH = (M::KIND == kModelFiveN);
    constexpr bool SXN = (M::KIND == kModelSixN);
    PT P[6][N];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        int x = i, y = j, z = k;
        if (d == 0) x += s - 3; else if (d == 1) y += s - 3; else z += s - 3;
        double Uc[N];
        const long long q = g.at(x, y, z);
#pragma unroll
        for (int c = 0; c < N; ++c) Uc[c] = U[c * g.S + q];
        if constexpr (MIX) M::cons2prim_f32(P[s], Uc, e);
        else M::cons2prim(P[s], Uc, e, nullptr);
    }
    double WfL[N], WfR[N], UL[N], UR[N];
    constexpr int NB0 = (SCHEME == 6) ? weno5b_plain_lo<M>() : 0;
    constexpr int NB1 = (SCHEME == 6) ? weno5b_plain_hi<M>() : N;
    double cm;
    if constexpr (!MIX) {
        if constexpr (SCHEME == 6 && (NPH || SXN)) {
            double rf[M::NP], af[M::NP];
            bounded_phases<M::NP, 5, double>([&](int k, int s) { return (double)P[s][M::IR + k]; },
                                         [&](int k, int s) { return (double)P[s][M::IA + k]; }, 1, rf, af);
            for (int k = 0; k < M::NP; ++k) { WfL[M::IR + k] = rf[k]; WfL[M::IA + k] = af[k]; }
            bounded_phases<M::NP, 5, double>([&](int k, int s) { return (double)P[s + 1][M::IR + k]; },
                                         [&](int k, int s) { return (double)P[s + 1][M::IA + k]; }, -1, rf, af);
            for (int k = 0; k < M::NP; ++k) { WfR[M::IR + k] = rf[k]; WfR[M::IA + k] = af[k]; }
        } else if constexpr (SCHEME == 6) {
            double r1[6], r2[6], al[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                r1[s] = P[s][0];
                r2[s] = P[s][1];
                al[s] = P[s][M::IA];
            }
            weno5b_masses(r1, r2, al, 1, WfL[0], WfL[1], WfL[M::IA]);
            weno5b_masses(r1 + 1, r2 + 1, al + 1, -1, WfR[0], WfR[1], WfR[M::IA]);
        }
        if constexpr (SCHEME == 2) {
#pragma unroll
            for (int n = 0; n < N; ++n) {
                WfL[n] = face3(P[1][n], P[2][n], P[3][n], dxd, 1, code);
                WfR[n] = face3(P[2][n], P[3][n], P[4][n], dxd, -1, code);
            }
            if (code == 11) {
                weno3b_faces<M, double>([&](int s, int n) { return P[1 + s][n]; }, 1, WfL);
                weno3b_faces<M, double>([&](int s, int n) { return P[2 + s][n]; }, -1, WfR);
            }
        } else {
#pragma unroll
            for (int n = NB0; n < NB1; ++n) {
                WfL[n] = weno5(P[0][n], P[1][n], P[2][n], P[3][n], P[4][n], 1);
                WfR[n] = weno5(P[1][n], P[2][n], P[3][n], P[4][n], P[5][n], -1);
            }
        }
        M::prim2cons(UL, WfL, e, err);
        M::prim2cons(UR, WfR, e, err);
        if constexpr (NPH && SCHEME != 6) if (SCHEME != 2 || code != 11) {
            M::consistent_limit(UL, P[2], 1, dxd, 1, e, err);
            M::consistent_limit(UR, P[3], 1, dxd, -1, e, err);
        }
        if constexpr (SXN && SCHEME == 2) if (code >= 1 && code < 10) {
            M::consistent_limit(UL, P[2], 1, dxd, 1, e, err);
            M::consistent_limit(UR, P[3], 1, dxd, -1, e, err);
        }
        riemann<M>(id_riemann, F, fnc, cm, UL, UR, e, d, id_k, err);
    } else {
        float wL[N], wR[N];
        if constexpr (SCHEME == 6 && NPH) {
            bounded_phases<M::NP, 5, float>([&](int k, int s) { return (float)P[s][k]; },
                                        [&](int k, int s) { return (float)P[s][M::IA + k]; }, 1, wL, wL + M::IA);
            bounded_phases<M::NP, 5, float>([&](int k, int s) { return (float)P[s + 1][k]; },
                                        [&](int k, int s) { return (float)P[s + 1][M::IA + k]; }, -1, wR, wR + M::IA);
        } else if constexpr (SCHEME == 6) {
            float r1[6], r2[6], al[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                r1[s] = P[s][0];
                r2[s] = P[s][1];
                al[s] = P[s][M::IA];
            }
            weno5b_masses_f32(r1, r2, al, 1, wL[0], wL[1], wL[M::IA]);
            weno5b_masses_f32(r1 + 1, r2 + 1, al + 1, -1, wR[0], wR[1], wR[M::IA]);
        }
        if constexpr (SCHEME == 2) {
#pragma unroll
            for (int n = 0; n < N; ++n) {
                wL[n] = face3_f32(P[1][n], P[2][n], P[3][n], 1, code);
                wR[n] = face3_f32(P[2][n], P[3][n], P[4][n], -1, code);
            }
            if (code == 11) {
                weno3b_faces<M, float>([&](int s, int n) { return (float)P[1 + s][n]; }, 1, wL);
                weno3b_faces<M, float>([&](int s, int n) { return (float)P[2 + s][n]; }, -1, wR);
            }
        } else {
#pragma unroll
            for (int n = NB0; n < NB1; ++n) {
                wL[n] = weno5_f32(P[0][n], P[1][n], P[2][n], P[3][n], P[4][n], 1);
                wR[n] = weno5_f32(P[1][n], P[2][n], P[3][n], P[4][n], P[5][n], -1);
            }
        }
#pragma unroll
        for (int n = 0; n < N; ++n) {
            WfL[n] = wL[n];
            WfR[n] = wR[n];
        }
        M::prim2cons(UL, WfL, e, err);
        M::prim2cons(UR, WfR, e, err);
        if constexpr (NPH) {
            if constexpr (SCHEME != 6) if (SCHEME != 2 || code != 11) {
                M::consistent_limit(UL, P[2], 1, dxd, 1, e, err);
                M::consistent_limit(UR, P[3], 1, dxd, -1, e, err);
            }
            riemann<M>(id_riemann, F, fnc, cm, UL, UR, e, d, id_k, err);
        } else if (id_riemann != 2) {
            float cmf;
            llf_hll_mixed<M>(id_riemann, F, fnc, cmf, UL, UR, wL, wR, e, d, id_k);
        } else {
            float cmf;
            if constexpr (M::KIND == kModelFive) fiveeq_hllc_mixed<D>(F, fnc, cmf, UL, UR, wL, wR, e, d, id_k);
            else sixeq_hllc_mixed<D>(F, fnc, cmf, UL, UR, wL, wR, e, d);
        }
    }
}

struct AmrCfArgs {
    const AmrCf* cf;
    int n;
    double* reg;
    double* reg_nc;
    AmrBufs B;
    const Grid* grids;  // per box
    int k;              // array of the stage input
    double w;           // the stage's dt share
    double dA[3];       // face areas of the level computing the fluxes
    Eos e;
    int id_k;
    int code;           // three-cell scheme code (SCHEME 2)
    int id_riemann;     // Physics.RiemannSolver
    double dx[3];       // cell sizes of the level computing the fluxes
    int role;           // 0: coarse (CrseInit, scale -w), 1: fine (FineAdd, scale w)
};

template <class M, int SCHEME, bool MIX>
__global__ void amr_cf_kernel(AmrCfArgs A) {
    constexpr int N = M::N, NC = M::NC;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < A.n; t += gridDim.x * blockDim.x) {
        const AmrCf& f = A.cf[t];
        const double dA = (f.d == 0) ? A.dA[0] : (f.d == 1 ? A.dA[1] : A.dA[2]);
        const double dxd = (f.d == 0) ? A.dx[0] : (f.d == 1 ? A.dx[1] : A.dx[2]);
        double F[N], fnc[NC];
        if (A.role == 0) {
            amr_face_flux<M, SCHEME, MIX>(A.B.p[f.cbox * 4 + A.k], A.grids[f.cbox], f.d, f.cface[0], f.cface[1],
                                          f.cface[2], A.e, A.id_k, A.code, A.id_riemann, dxd, F, fnc, nullptr);
            for (int c = 0; c < N; ++c) A.reg[(long long)t * N + c] += (-A.w) * (F[c] * dA);
            for (int c = 0; c < NC; ++c) A.reg_nc[(long long)t * NC + c] += (-A.w) * (fnc[c] * dA);
        } else {
            const int nf = (M::D == 3) ? 4 : 2;
            for (int a = 0; a < nf; ++a) {
                amr_face_flux<M, SCHEME, MIX>(A.B.p[f.fbox[a] * 4 + A.k], A.grids[f.fbox[a]], f.d, f.fface[a][0],
                                              f.fface[a][1], f.fface[a][2], A.e, A.id_k, A.code, A.id_riemann, dxd, F,
                                              fnc, nullptr);
                for (int c = 0; c < N; ++c) A.reg[(long long)t * N + c] += A.w * (F[c] * dA);
                for (int c = 0; c < NC; ++c) A.reg_nc[(long long)t * NC + c] += A.w * (fnc[c] * dA);
            }
        }
    }
}

// FluxRegister::Reflux and RefluxSourceTerms: one thread per coarse cell, its faces in list order.
// Five-equation model: alpha1 -= xi phi1 (1 + K1) (source/Class_Compressible5Eq_PhaseField.cpp:77-160).
// Six-equation model (source/Class_Compressible6Eq_PhaseField.cpp:85-195): the refluxed non-conservative
// face terms give div u, div(u a1p1), div(u a2p2) corrections, applied to the phase energies and alpha1
// with the primitives of the state before the reflux; with relax set, a cell the reflux changed is
// relaxed again (RelaxRefluxedCells, :314-349), since the stage relaxation preceded the reflux.
// N-phase six-equation model (source/Class_Compressible6Eq_IE_NPhase_PhaseField.cpp:83-181, :302-333):
// alpha_k -= alpha_k xi, alpha_k rho_k e_k += alpha_k p_k xi with xi the refluxed u* term and the
// primitives of the state before the reflux; the refluxed cells relaxed again likewise.
template <class M>
__global__ void amr_reflux_kernel(const AmrCf* cf, const int* groups, int ngroups, const double* reg,
                                  const double* reg_nc, AmrBufs B, int knew, double vol, Eos e, int id_k, int relax,
                                  double trace, unsigned int* err) {
    constexpr int N = M::N, NC = M::NC;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += gridDim.x * blockDim.x) {
        const int t0 = groups[gi], t1 = groups[gi + 1];
        const AmrCf& f0 = cf[t0];
        double* U = B.p[f0.cbox * 4 + knew];
        const long long S = B.S[f0.cbox];
        double Uc[N], W[N];
        for (int c = 0; c < N; ++c) Uc[c] = U[c * S + f0.cq];
        M::cons2prim(W, Uc, e, nullptr);
        double src = 0.0;
        double srck[(M::KIND == kModelFiveN) ? M::NP : 1];
        if constexpr (M::KIND == kModelFive) src = M::kapila_factor(Uc, W, e, id_k, nullptr);
        if constexpr (M::KIND == kModelFiveN) M::kapila_factors(srck, W, e, id_k, nullptr);
        double xs[NC];
        for (int t = t0; t < t1; ++t) {
            const double mult = cf[t].hi_side ? -1.0 : 1.0;
            for (int c = 0; c < N; ++c) U[c * S + f0.cq] += mult * reg[(long long)t * N + c] / vol;
            for (int c = 0; c < NC; ++c) {
                const double xi = mult * reg_nc[(long long)t * NC + c] / vol;
                xs[c] = (t == t0) ? xi : xs[c] + xi;
            }
        }
        if constexpr (M::KIND == kModelFive) {
            U[M::IA * S + f0.cq] += -1.0 * (xs[0] * src);
        } else if constexpr (M::KIND == kModelFiveN) {
            // source/Class_Compressible5Eq_NPhase_PhaseField.cpp:89-110: alpha_k -= xi phi_k (1 + K_k)
            for (int kk = 0; kk < M::NP; ++kk) U[(M::IA + kk) * S + f0.cq] += -1.0 * (srck[kk] * xs[0]);
        } else if constexpr (M::KIND == kModelSixN) {
            for (int kk = 0; kk < M::NP; ++kk) {
                U[(M::IA + kk) * S + f0.cq] += -W[M::IA + kk] * xs[0];
                U[(M::IP + kk) * S + f0.cq] += W[M::IP + kk] * xs[0];
            }
            if (relax) {
                double v[N];
                bool changed = false;
                for (int c = 0; c < N; ++c) {
                    v[c] = U[c * S + f0.cq];
                    changed = changed || (v[c] != Uc[c]);
                }
                if (changed) {
                    M::relax(v, e, trace, err);
                    for (int c = 0; c < N; ++c) U[c * S + f0.cq] = v[c];
                }
            }
        } else {
            const double divv = -xs[0], dva1 = -xs[1], dva2 = -xs[2];
            const double rho = W[0] + W[1];
            const double vg1 = dva1 - W[M::IE1] * divv;
            const double vg2 = dva2 - W[M::IE2] * divv;
            const double x = W[1] / rho * vg1 - W[0] / rho * vg2;
            U[M::IE1 * S + f0.cq] += x;
            U[M::IE2 * S + f0.cq] += -x;
            U[M::IA * S + f0.cq] += W[M::IA] * divv;
            if (relax) {
                double v[N];
                bool changed = false;
                for (int c = 0; c < N; ++c) {
                    v[c] = U[c * S + f0.cq];
                    changed = changed || (v[c] != Uc[c]);
                }
                if (changed) {
                    relax_pressure<M::D>(v, e, trace, err);
                    for (int c = 0; c < N; ++c) U[c * S + f0.cq] = v[c];
                }
            }
        }
    }
}

__global__ void amr_avg_kernel(const AmrAvg* t, long long n, AmrBufs B, int kc, int kf, int N, int nchild,
                               double volfrac) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const AmrAvg& e = t[q];
        double* C = B.p[e.cb * 4 + kc];
        const long long Sc = B.S[e.cb];
        for (int c = 0; c < N; ++c) {
            double s = 0.0;
            for (int h = 0; h < nchild; ++h) s += B.p[e.fb[h] * 4 + kf][c * B.S[e.fb[h]] + e.fq[h]];
            C[c * Sc + e.cq] = volfrac * s;
        }
    }
}

__global__ void amr_set_kernel(double* dt, double v, unsigned long long* cmax) {
    *dt = v;
    if (cmax) *cmax = 0ull;
}

}  // namespace compas
