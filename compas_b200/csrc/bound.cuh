// Bound-preserving right-hand side of the five-equation models (FiniteVolume.ID_Bound = 1): FIVEEQS and
// FIVEEQS_NPHASE, FP64 and the reference's arithmetic to the bit. The N-phase counterparts of the files
// below (include/Operators_Compressible5Eq_NPhase/, include/Physics_Compressible5Eq_NPhase/) have the
// same steps with sums over the phases; their MUSCL face states go through the consistent limiter
// (FVM_Reconstruction2Face_Conservative_MUSCL_D_Compressible5Eq_NPhase.H) and their WENO5B states bound
// every phase (FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq_NPhase.H).
//   flux functor branch          include/Operators_Compressible5Eq/FVM_Conservative2FluxHyperbolic_K_Compressible5Eq.H:100-152
//   MUSCLBP                      .../FVM_Reconstruction2FaceLR_Conservative_MUSCLBP_{K,D}_Compressible5Eq.H,
//                                .../FVM_Reconstruction2Face_Conservative_MUSCLBP_D_Compressible5Eq.H,
//                                .../FVM_Reconstruction2Face_Conservative_MUSCL_D_Compressible5Eq.H
//   WENO5BP                      .../FVM_Reconstruction2FaceLR_Conservative_WENO5BP_{K,D}_Compressible5Eq.H,
//                                .../FVM_Reconstruction2Face_Conservative_WENO5BP_D_Compressible5Eq.H,
//                                .../FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq.H:15-320
//   energy-bound limiter         .../FVM_Reconstruction2Face_Conservative_LimiterBound_Compressible5Eq.H,
//                                include/Operators_FV/Limiter_BoundMin.H, f_LimiterBound.H, fC_QuadratureRule.H
//   energy bound                 include/Physics_Compressible5Eq/Conservative2EnergyBound_Compressible5Eq.H,
//                                EquationOfState_Phase_Compressible5Eq.H (pressure base, internal energy)
//   HLL with bounded speeds      include/Physics_Compressible5Eq/Riemann_HLL_Bound_Compressible5Eq.H:16-137,
//                                Conservative2Lambda_HLL_Compressible5Eq.H, Conservative2A_Compressible5Eq.H,
//                                Conservative2Pmin_Compressible5Eq.H, Conservative2K_Compressible5Eq.H,
//                                NonConservative_Compressible5Eq.H
//   CFL speed                    include/Operators_Compressible5Eq/Conservative2CFLSpeed_HLL_Compressible5Eq.H
//   quadrature weights           include/Operators_FV/FiniteVolume_Parameter.H:60-173
//
// Layout. A stage is two kernels. bp_face_kernel computes every face of the box, one thread per face,
// in the face layout of compas_b200_face_fluxes (direction d: (n_d + 1) faces along d, x fastest): the
// N fluxes and the normal face velocity (the non-conservative face quantity FluxNC[0]). A face needs
// the limited right-face state of its left cell and the limited left-face state of its right cell;
// the energy-bound limiter of a cell needs both of its face states, so each thread reconstructs its two
// cells completely (twice the reconstruction work of a cell-centred pass; the bounded-speed HLL solver,
// with its four wave-speed bounds and two CFL speeds, costs more than both reconstructions). The
// stencil cells are read from global memory: neighbouring threads read neighbouring cells, so the
// loads coalesce and the reuse hits L1/L2. bp_update_kernel forms the divergence of the face fluxes and
// the non-conservative term cell by cell, the Runge-Kutta combination, and the smallest energy bound of
// the new stage state (MinEnergyBound, source/Class_Compressible_PhaseField.cpp:3596-3635), which the
// host reads to decide whether the step has to be taken again.
#pragma once

namespace compas {

// Arguments of the bound-preserving face pass.
struct BpFaceArgs {
    const double* U;          // stage state, ghosts filled
    Grid g;
    Eos e;
    int D;
    int physics, nphase;      // model of the launch (COMPAS_B200_FIVEEQS or _FIVEEQS_NPHASE, NPHASE)
    int weno;                 // 1 WENO5BP (WENO3, WENO3B, WENO5, WENO5B), 0 MUSCLBP
    int lim;                  // MUSCLBP limiter (ID_Limiter 0..4)
    int id_k;                 // Physics.source_term
    int id_lambda;            // 1 the sound speed (ID_Lambda special), 0 the general bound
    double wb;                // quadrature weight of the limiters (1/6, or 1/12 for WENO5 / WENO5B)
    double qw;                // Quadrature_Weight of the CFL speed (1, 1/6 or 1/12)
    double dx[3];
    double area[3];           // face-flux scale (1, or the face areas of ScaleFaceFluxesByArea)
    long long off[4];         // first thread of each direction's faces
    double* F[3];             // N face fluxes per direction (may be null: wave speeds only)
    double* V[3];             // normal face velocity per direction (may be null)
    int which;                // COMPAS_B200_FACES_ALL or COMPAS_B200_FACES_BOUNDARY
    const int* done;          // device flag: nothing to do when set (may be null)
    const unsigned long long* prev_eb;  // energy-bound keys of the earlier stages of the step: nothing to do
    int nprev;                          // when one of them is < 0 (the step is taken again)
    unsigned long long* cmax; // double bits, atomicMax (may be null)
    unsigned int* err;
};

// Arguments of the bound-preserving stage update.
struct BpUpdateArgs {
    const double* Us;         // stage state
    const double* U0;         // state at the start of the step (stages 1, 2)
    double* Uout;             // new state (mode kModeStage) or dUdt (kModeDudt)
    Grid g;
    Eos e;
    int D;
    int physics, nphase;
    int mode;
    int stage;
    int id_k;
    const double* dt;         // device scalar
    double dx[3];
    const double* F[3];
    const double* V[3];
    const int* done;
    const unsigned long long* prev_eb;
    int nprev;
    unsigned long long* eb;   // smallest energy bound of the new state, as an ordered key (atomicMin)
    unsigned int* err;
};

// Ordered keys of doubles: key(a) < key(b) exactly when a < b (for non-NaN values; -0 < +0), so that
// an unsigned 64-bit atomicMin gives the smallest value.
__device__ __forceinline__ unsigned long long bp_key(double x) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ bool bp_key_negative(unsigned long long k) {
    // keys of negative doubles (and of -0) have the top bit clear; -0 is not < 0
    return !(k >> 63) && k != 0x7fffffffffffffffull;
}
__device__ __forceinline__ bool bp_earlier_failed(const unsigned long long* prev, int n) {
    for (int q = 0; q < n; ++q)
        if (bp_key_negative(prev[q])) return true;
    return false;
}

// Conservative2EnergyBound: rho E - |rho u|^2 / (2 rho) - sum_k (phi_k A_k p_min,k + phi_k B_k + alpha_k rho_k D_k).
template <class M>
__device__ __forceinline__ double bp_energy_bound(const double* U, const Eos& e, unsigned int* err) {
    constexpr int D = M::D;
    if constexpr (M::KIND == kModelFive) {
        const double a1r1 = U[0], a2r2 = U[1], rhoE = U[M::IE], alpha1 = U[M::IA];
        const double alpha2 = 1.0 - alpha1;
        const double rho = a1r1 + a2r2;
        const double phi1 = nasg_phi(alpha1, a1r1, e.C1, err);
        const double e1 = ((phi1 * e.A1) * e.pmin1 + phi1 * e.B1) + a1r1 * e.D1;
        const double phi2 = nasg_phi(alpha2, a2r2, e.C2, err);
        const double e2 = ((phi2 * e.A2) * e.pmin2 + phi2 * e.B2) + a2r2 * e.D2;
        const double rho_e_min = e1 + e2;
        const double m2 = ksum<D>(U + M::IM);
        return (rhoE - (0.5 * m2) / rho) - rho_e_min;
    } else {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < M::NP; ++k) rho += U[k];
        double rho_e_min = 0.0;
#pragma unroll
        for (int k = 0; k < M::NP; ++k) {
            const double phi = nasg_phi(U[M::IA + k], U[k], e.Ck[k], err);
            rho_e_min += ((phi * e.Ak[k]) * e.pmink[k] + phi * e.Bk[k]) + U[k] * e.Dk[k];
        }
        const double m2 = ksum<D>(U + M::IM);
        return (U[M::IE] - (0.5 * m2) / rho) - rho_e_min;
    }
}

// NonConservative: K_k = rho c^2 / (rho_k c_k^2) - 1 with the Wood mixture (source_term 1), 0 otherwise,
// from the primitives W.
template <class M>
__device__ __forceinline__ void bp_K(const double* W, const Eos& e, int id_k, double* K, unsigned int* err) {
    if (id_k != 1) {
#pragma unroll
        for (int k = 0; k < M::NP; ++k) K[k] = 0.0;
        return;
    }
    if constexpr (M::KIND == kModelFive) {
        const double p = W[M::IE], alpha1 = W[M::IA];
        const double r1c1 = ((e.A1 + 1.0) * p + e.B1) / e.A1;
        const double r2c2 = ((e.A2 + 1.0) * p + e.B2) / e.A2;
        const double alpha2 = 1.0 - alpha1;
        const double ph1 = nasg_phi(alpha1, W[0], e.C1, err);
        const double ph2 = nasg_phi(alpha2, W[1], e.C2, err);
        const double rho_c2 = 1.0 / (ph1 / r1c1 + ph2 / r2c2);
        K[0] = rho_c2 / r1c1 - 1.0;
        K[1] = rho_c2 / r2c2 - 1.0;
    } else {
        double rc2[M::NP];
#pragma unroll
        for (int k = 0; k < M::NP; ++k) rc2[k] = M::rc2_phase(W[M::IE], e, k);
        const double rho_c2 = M::rho_c2_mix(W, rc2, e, 1, err);
#pragma unroll
        for (int k = 0; k < M::NP; ++k) K[k] = rho_c2 / rc2[k] - 1.0;
    }
}

// What the bounded speeds need of a cell state U0 next to the face: Conservative2A, Conservative2Pmin
// and the largest |1 + K_k| of Conservative2CFLSpeed_HLL, from one primitive conversion.
struct BpCell {
    double A, Pmin, kmax;
};
template <class M>
__device__ __forceinline__ BpCell bp_cell(const double* U0, const Eos& e, int id_k, unsigned int* err) {
    double W[M::N], K[M::NP];
    M::cons2prim(W, U0, e, err);
    bp_K<M>(W, e, id_k, K, err);
    BpCell c;
    if constexpr (M::KIND == kModelFive) {
        const double alpha1 = W[M::IA], alpha2 = 1.0 - alpha1;
        const double phi1 = (id_k == 1) ? nasg_phi(alpha1, W[0], e.C1, err) : alpha1;
        const double phi2 = (id_k == 1) ? nasg_phi(alpha2, W[1], e.C2, err) : alpha2;
        const double f1 = phi1 * (1.0 + K[0]), f2 = phi2 * (1.0 + K[1]);
        c.A = f1 * ((e.A1 + 1.0) * e.pmin1 + e.B1) + f2 * ((e.A2 + 1.0) * e.pmin2 + e.B2);
        c.Pmin = f1 * e.pmin1 + f2 * e.pmin2;
        c.kmax = dmax(dmax(0.0, fabs(1.0 + K[0])), fabs(1.0 + K[1]));
    } else {
        c.A = 0.0;
        c.Pmin = 0.0;
        c.kmax = 0.0;
#pragma unroll
        for (int k = 0; k < M::NP; ++k) {
            const double al = W[M::IA + k];
            const double phi = (id_k == 1) ? nasg_phi(al, W[k], e.Ck[k], err) : al;
            const double f = phi * (1.0 + K[k]);
            c.A += f * ((e.Ak[k] + 1.0) * e.pmink[k] + e.Bk[k]);
            c.Pmin += f * e.pmink[k];
            c.kmax = dmax(c.kmax, fabs(1.0 + K[k]));
        }
    }
    return c;
}

// Density of the primitives W (Primitive2State's partial densities summed as the reference does).
template <class M>
__device__ __forceinline__ double bp_rho(const double* W) {
    if constexpr (M::KIND == kModelFive) {
        return W[0] + W[1];
    } else {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < M::NP; ++k) rho += W[k];
        return rho;
    }
}

// Both energy-bounded face states of the cell at (i, j, k): Ufp at its right face, Ufm at its left
// face along d, in conservative variables. The stencil along d is read from U: cells -1..+1 (MUSCLBP)
// or -2..+2 (WENO5BP).
template <class M>
__device__ __forceinline__ void bp_cell_faces(const BpFaceArgs& a, int d, int i, int j, int k, double* Ufp,
                                              double* Ufm, unsigned int* err) {
    constexpr int N = M::N, D = M::D, IA = M::IA;
    constexpr bool NPH = (M::KIND == kModelFiveN);
    const Grid& g = a.g;
    const long long q0 = g.at(i, j, k);
    const long long sd = (d == 0) ? 1 : (d == 1 ? g.px : g.pxy);
    double Uc[N];
    load_cons<M>(Uc, a.U, g, q0);
    double Wp[N], Wm[N];
    if (a.weno) {
        double W[5][N];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            double Us[N];
            load_cons<M>(Us, a.U, g, q0 + (s - 2) * sd);
            M::cons2prim(W[s], Us, a.e, err);
        }
        if constexpr (NPH) {
            double rf[M::NP], af[M::NP];
            auto r = [&](int kk, int s) { return W[s][kk]; };
            auto al = [&](int kk, int s) { return W[s][IA + kk]; };
            bounded_phases<M::NP, 5, double>(r, al, 1, rf, af, a.wb);
#pragma unroll
            for (int kk = 0; kk < M::NP; ++kk) { Wp[kk] = rf[kk]; Wp[IA + kk] = af[kk]; }
            bounded_phases<M::NP, 5, double>(r, al, -1, rf, af, a.wb);
#pragma unroll
            for (int kk = 0; kk < M::NP; ++kk) { Wm[kk] = rf[kk]; Wm[IA + kk] = af[kk]; }
        } else {
            double r1[5], r2[5], al[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                r1[s] = W[s][0];
                r2[s] = W[s][1];
                al[s] = W[s][IA];
            }
            weno5b_masses_both(r1, r2, al, a.wb, Wp, Wm, IA);
        }
        // velocity and pressure(s) by plain WENO5
#pragma unroll
        for (int n = M::IM; n < IA; ++n) {
            Wp[n] = weno5(W[0][n], W[1][n], W[2][n], W[3][n], W[4][n], 1);
            Wm[n] = weno5(W[0][n], W[1][n], W[2][n], W[3][n], W[4][n], -1);
        }
        M::prim2cons(Ufp, Wp, a.e, err);
        M::prim2cons(Ufm, Wm, a.e, err);
    } else {
        double W[3][N];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            if (s == 1) {
                M::cons2prim(W[s], Uc, a.e, err);
            } else {
                double Us[N];
                load_cons<M>(Us, a.U, g, q0 + (s - 1) * sd);
                M::cons2prim(W[s], Us, a.e, err);
            }
        }
        const double dxd = pick<D>(a.dx, d);
#pragma unroll
        for (int n = 0; n < N; ++n) {
            Wp[n] = muscl_face(W[0][n], W[1][n], W[2][n], dxd, 1, a.lim);
            Wm[n] = muscl_face(W[0][n], W[1][n], W[2][n], dxd, -1, a.lim);
        }
        M::prim2cons(Ufp, Wp, a.e, err);
        M::prim2cons(Ufm, Wm, a.e, err);
        if constexpr (NPH) {
            // the N-phase MUSCL face state goes through the consistent limiter about the cell
            M::consistent_limit(Ufp, W[1], 1, dxd, 1, a.e, err);
            M::consistent_limit(Ufm, W[1], 1, dxd, -1, a.e, err);
        }
    }
    // energy-bound limiter about the cell average (LimiterBound with Limiter_BoundMin, lower bound 0)
    const double w = a.wb;
    double C[N];
#pragma unroll
    for (int n = 0; n < N; ++n) C[n] = ((Uc[n] - w * Ufp[n]) - w * Ufm[n]) / (1.0 - 2.0 * w);
    const double eb_c = bp_energy_bound<M>(Uc, a.e, err);
    const double eb_C = bp_energy_bound<M>(C, a.e, err);
    const double eb_p = bp_energy_bound<M>(Ufp, a.e, err);
    const double eb_m = bp_energy_bound<M>(Ufm, a.e, err);
    double mn = eb_C;  // std::min({fC, fL_fp, fR_fm})
    if (eb_p < mn) mn = eb_p;
    if (eb_m < mn) mn = eb_m;
    const double th = dmin(1.0, dmax(0.0, eb_c - 0.0) / dmax(0.0, eb_c - mn));
#pragma unroll
    for (int n = 0; n < N; ++n) {
        Ufp[n] = Uc[n] + th * (Ufp[n] - Uc[n]);
        Ufm[n] = Uc[n] + th * (Ufm[n] - Uc[n]);
    }
}

// Conservative2Lambda_HLL of the face state U (primitives W, sound speed c, energy bound eb) about the
// cell state described by b.
template <class M>
__device__ __forceinline__ void bp_lambda(const double* W, double c, double eb, const BpCell& b, int d, int id_lambda,
                                          double& lp, double& lm) {
    const double V = pick<M::D>(W + M::IM, d);
    double C = c;
    if (id_lambda == 0 || isnan(c)) {
        const double rho = bp_rho<M>(W);
        C = dmax(fabs((W[M::IE] - b.Pmin) + b.A) / sqrt((2.0 * rho) * eb), c);
    }
    lp = V + C;
    lm = V - C;
}

// One face: fluxes F, the normal face velocity and the face's CFL speed (the flux functor's cmax).
// (fi, fj, fk) is the cell on the high side of the face.
template <class M>
__device__ __forceinline__ void bp_face(const BpFaceArgs& a, int d, int fi, int fj, int fk, double* F, double& vel,
                                        double& cm, unsigned int* err) {
    constexpr int N = M::N, D = M::D;
    const int li = fi - (d == 0), lj = fj - (d == 1), lk = fk - (d == 2);
    double UL[N], UR[N];
    {
        double other[N];
        bp_cell_faces<M>(a, d, li, lj, lk, UL, other, err);
        bp_cell_faces<M>(a, d, fi, fj, fk, other, UR, err);
    }
    double Um[N], Uc[N];
    load_cons<M>(Um, a.U, a.g, a.g.at(li, lj, lk));
    load_cons<M>(Uc, a.U, a.g, a.g.at(fi, fj, fk));
    const BpCell bm = bp_cell<M>(Um, a.e, a.id_k, err);
    const BpCell bc = bp_cell<M>(Uc, a.e, a.id_k, err);
    double WL[N], WR[N];
    M::cons2prim(WL, UL, a.e, err);
    M::cons2prim(WR, UR, a.e, err);
    const double cL = M::sound_speed(WL, a.e, a.id_k, err);
    const double cR = M::sound_speed(WR, a.e, a.id_k, err);
    // the energy bounds of the face states enter the general speed bound only
    const double ebL = (a.id_lambda == 0 || isnan(cL)) ? bp_energy_bound<M>(UL, a.e, err) : 0.0;
    const double ebR = (a.id_lambda == 0 || isnan(cR)) ? bp_energy_bound<M>(UR, a.e, err) : 0.0;
    double lLLp, lLLm, lLRp, lLRm, lRLp, lRLm, lRRp, lRRm;
    bp_lambda<M>(WL, cL, ebL, bm, d, a.id_lambda, lLLp, lLLm);
    bp_lambda<M>(WL, cL, ebL, bc, d, a.id_lambda, lLRp, lLRm);
    bp_lambda<M>(WR, cR, ebR, bm, d, a.id_lambda, lRLp, lRLm);
    bp_lambda<M>(WR, cR, ebR, bc, d, a.id_lambda, lRRp, lRRm);
    const double lLp = dmax(lLLp, lLRp), lLm = dmin(lLLm, lLRm);
    const double lRp = dmax(lRLp, lRRp), lRm = dmin(lRLm, lRRm);
    const double Sp = dmax(dmax(0.0, lLp), lRp) + 1.0e-10;
    const double Sm = dmin(dmin(0.0, lLm), lRm) - 1.0e-10;
    vel = (Sp * pick<D>(WL + M::IM, d) - Sm * pick<D>(WR + M::IM, d)) / (Sp - Sm);
    double FL[N], FR[N];
    M::flux(FL, UL, WL, d);
    M::flux(FR, UR, WR, d);
#pragma unroll
    for (int n = 0; n < N; ++n) F[n] = ((Sp * FL[n] - Sm * FR[n]) + (Sp * Sm) * (UR[n] - UL[n])) / (Sp - Sm);
    const double c = dmax(-Sm, Sp);
    const double cfl_c = 2.0 * (c + (a.qw * bc.kmax) * c);
    const double cfl_m = 2.0 * (c + (a.qw * bm.kmax) * c);
    cm = dmax(cfl_c, cfl_m);
}

// Every face of the box (or its boundary faces), one thread each; fluxes (times area[d]) and the normal
// face velocity into the face arrays, the largest CFL speed of the faces on the low side of the valid
// cells into *cmax.
template <class M>
__global__ void __launch_bounds__(128) bp_face_kernel(BpFaceArgs a) {
    constexpr int N = M::N, D = M::D;
    if (a.done && *a.done) return;
    if (bp_earlier_failed(a.prev_eb, a.nprev)) return;
    const long long total = a.off[D];
    double cml = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int d = 0;
        while (d + 1 < D && t >= a.off[d + 1]) ++d;
        long long r = t - a.off[d];
        const long long e0 = a.g.n[0] + (d == 0), e1 = a.g.n[1] + (d == 1), e2 = (D == 3) ? a.g.n[2] + (d == 2) : 1;
        long long f[3];
        if (a.which == 0) {
            f[0] = r % e0;
            f[1] = (r / e0) % e1;
            f[2] = r / (e0 * e1);
        } else {
            const int side = (int)(r & 1);
            r >>= 1;
            const int ax = (d == 0) ? 1 : 0, bx = (d == 2) ? 1 : 2;
            const long long ea = (ax == 0) ? e0 : e1;
            f[d] = side ? a.g.n[d] : 0;
            f[ax] = r % ea;
            f[bx] = (D == 3) ? r / ea : 0;
        }
        double F[N], vel, cm;
        bp_face<M>(a, d, (int)f[0], (int)f[1], (int)f[2], F, vel, cm, a.err);
        const long long q = f[0] + e0 * (f[1] + e1 * f[2]), S = e0 * e1 * e2;
        if (a.F[d]) {
            const double s = a.area[d];
#pragma unroll
            for (int n = 0; n < N; ++n) a.F[d][n * S + q] = (s == 1.0) ? F[n] : F[n] * s;
        }
        if (a.V[d]) a.V[d][q] = (a.area[d] == 1.0) ? vel : vel * a.area[d];
        if (f[d] < a.g.n[d]) cml = dmax(cm, cml);
    }
    if (a.cmax) {
        double v = cml;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) atomicMax(a.cmax, (unsigned long long)__double_as_longlong(v));
    }
}

// Divergence of the face fluxes (the reference's FVM_SurfaceIntegral: (F_high - F_low)/dx per
// direction, summed x, y, z) and alpha_k += phi_k (1 + K_k) div u* (FVM_SurfaceIntegralNC_Compressible5Eq.H,
// the N-phase one per phase), then the stage combination of ThirdOrderSSPRK and the new state's
// energy bound.
template <class M>
__global__ void __launch_bounds__(128) bp_update_kernel(BpUpdateArgs a) {
    constexpr int N = M::N, D = M::D, IA = M::IA;
    if (a.done && *a.done) return;
    if (bp_earlier_failed(a.prev_eb, a.nprev)) return;
    const Grid& g = a.g;
    const long long nx = g.n[0], ny = g.n[1], nz = (D == 3) ? g.n[2] : 1;
    const long long cells = nx * ny * nz;
    double dt = 0.0, ca = 1.0, cb = 0.0, cd = 1.0;
    if (a.mode == kModeStage) {
        dt = *a.dt;
        if (a.stage == 1) { ca = 0.25; cb = 0.75; cd = 0.25; }
        else if (a.stage == 2) { ca = 2.0 / 3.0; cb = 1.0 / 3.0; cd = 2.0 / 3.0; }
    }
    const double sdt = cd * dt;
    unsigned long long kmin = ~0ull;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / (nx * ny));
        double acc[N + 1];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const long long e0 = nx + (d == 0), e1 = ny + (d == 1), e2 = (D == 3) ? nz + (d == 2) : 1;
            const long long S = e0 * e1 * e2;
            const long long ql = i + e0 * (j + e1 * (long long)k);
            const long long qh = ql + ((d == 0) ? 1 : (d == 1 ? e0 : e0 * e1));
            const double dxd = a.dx[d];
#pragma unroll
            for (int c = 0; c <= N; ++c) {
                const double df = (c < N) ? a.F[d][c * S + qh] - a.F[d][c * S + ql] : a.V[d][qh] - a.V[d][ql];
                const double tt = df / dxd;
                acc[c] = (d == 0) ? tt : acc[c] + tt;
            }
        }
        const long long q = g.at(i, j, k);
        double Us[N], W[N], L[N];
        load_cons<M>(Us, a.Us, g, q);
        M::cons2prim(W, Us, a.e, a.err);
#pragma unroll
        for (int n = 0; n < N; ++n) L[n] = -acc[n];
        if constexpr (M::KIND == kModelFive) {
            const double fac = M::kapila_factor(W, W, a.e, a.id_k, a.err);
            L[IA] = L[IA] + fac * acc[N];
        } else {
            double fac[M::NP];
            M::kapila_factors(fac, W, a.e, a.id_k, a.err);
#pragma unroll
            for (int k = 0; k < M::NP; ++k) L[IA + k] = L[IA + k] + fac[k] * acc[N];
        }
        double out[N];
        if (a.mode == kModeDudt) {
#pragma unroll
            for (int n = 0; n < N; ++n) out[n] = L[n];
        } else {
            if (a.stage == 0) {
#pragma unroll
                for (int n = 0; n < N; ++n) out[n] = 1.0 * Us[n] + sdt * L[n];
            } else {
                double U0[N];
                load_cons<M>(U0, a.U0, g, q);
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const double v = ca * Us[n] + cb * U0[n];
                    out[n] = v + sdt * L[n];
                }
            }
            bool bad = false;
#pragma unroll
            for (int n = 0; n < N; ++n) bad |= isnan(out[n]);
            if (bad) flag_error(a.err, COMPAS_B200_ERR_NAN);
            const double eb = bp_energy_bound<M>(out, a.e, a.err);
            if (!isnan(eb)) {
                const unsigned long long kk = bp_key(eb);
                if (kk < kmin) kmin = kk;
            }
        }
#pragma unroll
        for (int n = 0; n < N; ++n) a.Uout[n * g.S + q] = out[n];
    }
    if (a.eb) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, kmin, o);
            if (v < kmin) kmin = v;
        }
        if ((threadIdx.x & 31) == 0 && kmin != ~0ull) atomicMin(a.eb, kmin);
    }
}

// Smallest energy bound of the valid cells (MinEnergyBound) as an ordered key.
template <class M>
__global__ void __launch_bounds__(128) bp_min_kernel(const double* U, Grid g, Eos e, unsigned long long* key,
                                                     unsigned int* err) {
    constexpr int D = M::D;
    const long long nx = g.n[0], ny = g.n[1], cells = nx * ny * (D == 3 ? g.n[2] : 1);
    unsigned long long kmin = ~0ull;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / (nx * ny));
        double Uc[M::N];
        load_cons<M>(Uc, U, g, g.at(i, j, k));
        const double eb = bp_energy_bound<M>(Uc, e, err);
        if (!isnan(eb)) {
            const unsigned long long kk = bp_key(eb);
            if (kk < kmin) kmin = kk;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, kmin, o);
        if (v < kmin) kmin = v;
    }
    if ((threadIdx.x & 31) == 0 && kmin != ~0ull) atomicMin(key, kmin);
}

}  // namespace compas
