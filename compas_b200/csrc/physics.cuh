// Pointwise physics of the two-phase diffuse-interface models on the device: state layout,
// conservative <-> primitive conversion through the stiffened-gas / NASG EOS, sound speed, WENO5
// face values, the HLLC flux and the six-equation pressure relaxation.
//
// The plain FP64 path must reproduce the reference arithmetic to the bit, so every formula below is
// evaluated with the same operations in the same association as the reference (C++ evaluates a+b+c
// as (a+b)+c and a*b*c as (a*b)*c), and the library is compiled with FMA contraction off. Where a
// value is recomputed several times in the reference from the same inputs it is computed once here:
// the result is the same double.
//
// Reference correspondence (file:line in the reference tree):
//   state layout           include/Physics_Compressible5Eq/Variables_Compressible5Eq.H:16-25
//                          include/Physics_Compressible6Eq/Variables_Compressible6Eq.H:16-26
//   NASG covolume          include/EquationOfState_NASG.H:26-58
//   5Eq C2P / P2C / EOS    include/Physics_Compressible5Eq/Conservative2Primitive_Compressible5Eq.H:15-61,
//                          Primitive2Conservative_Compressible5Eq.H, EquationOfState_Mixture_Compressible5Eq.H:15-77
//   5Eq sound speed        SoundSpeed_Compressible5Eq.H, rho_c2_Mixture_Compressible5Eq.H, rho_c2_Phase_Compressible5Eq.H
//   6Eq C2P / P2C / EOS    include/Physics_Compressible6Eq/Conservative2Primitive_Compressible6Eq.H:15-80,
//                          Primitive2Conservative_Compressible6Eq.H, EquationOfState_Phase_Compressible6Eq.H:15-73
//   6Eq sound speed        SoundSpeed_Compressible6Eq.H, rho_c2_Phase_Compressible6Eq.H, rho_c2_Mixture_Compressible6Eq.H
//   WENO5                  include/Operators_FV/WENO5.H:12-75, Reconstruction2Face_WENO.H
//   HLLC                   include/Physics_Compressible5Eq/Riemann_HLLC_Compressible5Eq.H:16-194
//                          include/Physics_Compressible6Eq/Riemann_HLLC_Compressible6Eq.H:16-255
//   relaxation             include/Physics_Compressible6Eq/Relaxation_Pressure_Instantaneous_Compressible6Eq.H:32-220
//                          include/RelaxationPressure_Safeguarded.H:17-256
#pragma once

#include <cfloat>
#include <cstdint>

#include "compas_b200.h"

namespace compas {

// Error bits of the per-run status word (compas_b200.h: COMPAS_B200_ERR_*).
__device__ __forceinline__ void flag_error(unsigned int* err, unsigned int bit) {
    if (err) atomicOr(err, bit);
}

// Reference semantics of std::min / std::max (first argument returned on ties and NaN second).
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double sgn0(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// Reciprocal for the mixed-precision form: an FP32 estimate refined by one Newton-Raphson step for
// 1/x, r1 = r0 (2 - x r0), evaluated in FP64 (Newton's method; the relative error squares, from
// about 2^-22 to below 2^-43). For x of FP32 range (densities, A_P). The quantities scaled by it are
// rounded to FP32 afterwards, so the result matches the IEEE FP64 quotient except within 2^-43 of a
// rounding boundary, at a fraction of the cost of an FP64 division.
__device__ __forceinline__ double rcp_mixed(double x) {
    const double r0 = (double)__fdividef(1.0f, (float)x);
    return r0 * (2.0 - x * r0);
}

// EOS coefficients, partial form alpha rho e = A Pi + B phi + alpha rho D, with C the NASG covolume b
// (source/Parm.cpp:101-188): the two phases of FIVEEQS / SIXEQS, and the per-phase lists of
// FIVEEQS_NPHASE (source/Parm.cpp:185-262).
constexpr int kMaxPhases = COMPAS_B200_MAX_PHASES;
struct Eos {
    double A1, A2, B1, B2, C1, C2, D1, D2;
    double iA1, iA2;  // 1/A1, 1/A2 (mixed-precision pressure recovery)
    double pinf1, pinf2;  // B1/(A1 + 1), B2/(A2 + 1) (the relaxation's admissibility check)
    double pmin1, pmin2;  // p_min of the two-phase Parm (source/Parm.cpp:164-171): -B/A, or -B/(A + 1) with K
    double Ak[kMaxPhases], Bk[kMaxPhases], Ck[kMaxPhases], Dk[kMaxPhases];
    double pmink[kMaxPhases];  // p_min of the N-phase Parm, the same rule per phase (source/Parm.cpp:255-261)
    // FP32 copies (round to nearest) of A, B, C of the two phases for the mixed form's FP32 wave speeds,
    // so that the face loop converts no coefficients
    float fA1, fA2, fB1, fB2, fC1, fC2;
};

// Model families of the stage kernel (the M::KIND of each model struct).
enum { kModelFive = 0, kModelSix = 1, kModelFiveN = 2, kModelSixN = 3 };

// NASG: phi = alpha - b alpha rho (alpha when b = 0); covolume violation 1 - b rho <= 0 is reported
// through the status word where the reference aborts.
__device__ __forceinline__ double nasg_phi(double alpha, double alpha_rho, double b, unsigned int* err) {
    if (b > 0.0 && alpha > 0.0) {
        const double xi = 1.0 - b * (alpha_rho / alpha);
        if (!(xi > 0.0)) flag_error(err, COMPAS_B200_ERR_COVOLUME);
    }
    return (b > 0.0) ? alpha - b * alpha_rho : alpha;
}
__device__ __forceinline__ double nasg_xi(double alpha, double alpha_rho, double b, unsigned int* err) {
    if (b > 0.0 && alpha > 0.0) {
        const double xi = 1.0 - b * (alpha_rho / alpha);
        if (!(xi > 0.0)) flag_error(err, COMPAS_B200_ERR_COVOLUME);
        return xi;
    }
    return 1.0;
}

// NASG covolume factor from a phase density (THINC face states): 1 - b rho, 1 when b = 0
// (include/EquationOfState_NASG.H:52-57).
__device__ __forceinline__ double nasg_xi_rho(double rho, double b, unsigned int* err) {
    if (b > 0.0) {
        const double xi = 1.0 - b * rho;
        if (!(xi > 0.0)) flag_error(err, COMPAS_B200_ERR_COVOLUME);
        return xi;
    }
    return 1.0;
}

// FiniteVolume.THINC parameters (include/Operators_FV/FiniteVolume_Parameter.H:34-38, 175-180).
struct Thinc {
    int use_normal;   // FiniteVolume.THINC.UseNormal
    double eps;       // FiniteVolume.THINC.EPS
    double beta;      // FiniteVolume.THINC.Beta
    double thr;       // FiniteVolume.THINC.NormalThreshold
};

// v[d] for a run-time direction d without indexing a per-thread array by a run-time value (which
// would place the array in local memory).
template <int D>
__device__ __forceinline__ double pick(const double* v, int d) {
    if (D == 2) return (d == 0) ? v[0] : v[1];
    return (d == 0) ? v[0] : ((d == 1) ? v[1] : v[2]);
}

template <int D>
__device__ __forceinline__ double ksum(const double* u) {
    // u*u + v*v (+ w*w), left to right
    double s = u[0] * u[0] + u[1] * u[1];
    if (D == 3) s = s + u[2] * u[2];
    return s;
}

// ------------------------------------------------------------------------------------------------
// Five-equation model: U = (a1r1, a2r2, rho u_d, rho E, alpha1), W = (a1r1, a2r2, u_d, p, alpha1)
// ------------------------------------------------------------------------------------------------
template <int DIM>
struct FiveEq {
    static constexpr int KIND = kModelFive;
    static constexpr int D = DIM;
    static constexpr int N = 4 + DIM;
    static constexpr int NC = 1;       // face quantities of the non-conservative terms
    static constexpr int NCPF = 1;     // of the Phase-Field step (none: FluxNC stays 0)
    static constexpr int NP = 2;        // phases
    static constexpr int IM = 2;        // rho u_d (u_d among the primitives)
    static constexpr int IE = 2 + DIM;  // total energy
    static constexpr int IA = 3 + DIM;  // alpha1

    __device__ static __forceinline__ void cons2prim(double* W, const double* U, const Eos& e, unsigned int* err) {
        const double a1r1 = U[0], a2r2 = U[1], alpha1 = U[IA];
        const double rho = a1r1 + a2r2;
        double u[3];
        for (int d = 0; d < D; ++d) u[d] = U[2 + d] / rho;
        const double rho_e = U[IE] - (0.5 * rho) * ksum<D>(u);
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = nasg_phi(alpha1, a1r1, e.C1, err);
        const double phi2 = nasg_phi(alpha2, a2r2, e.C2, err);
        const double rho_D = a1r1 * e.D1 + a2r2 * e.D2;
        const double AP = phi1 * e.A1 + phi2 * e.A2;
        const double BP = phi1 * e.B1 + phi2 * e.B2;
        W[0] = a1r1;
        W[1] = a2r2;
        for (int d = 0; d < D; ++d) W[2 + d] = u[d];
        W[IE] = ((rho_e - rho_D) - BP) / AP;
        W[IA] = alpha1;
    }

    // Mixed precision: primitives rounded to FP32 for the reconstruction. The pressure numerator
    // rho e - rho D - B_P, where the energy cancels against alpha B (~1e9), is formed in FP64; the
    // divisions (velocities, the well-conditioned A_P) run in FP32.
    __device__ static __forceinline__ void cons2prim_f32(float* W, const double* U, const Eos& e) {
        const double a1r1 = U[0], a2r2 = U[1], alpha1 = U[IA];
        const double rho = a1r1 + a2r2;
        const double ir = rcp_mixed(rho);  // near-FP64 reciprocal: u = fl32(rho u / rho) keeps uniform flow uniform
        double m2 = U[2] * U[2] + U[3] * U[3];
        if (D == 3) m2 += U[4] * U[4];
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = (e.C1 > 0.0) ? alpha1 - e.C1 * a1r1 : alpha1;
        const double phi2 = (e.C2 > 0.0) ? alpha2 - e.C2 * a2r2 : alpha2;
        const double num = ((U[IE] - 0.5 * m2 * ir) - (a1r1 * e.D1 + a2r2 * e.D2)) - (phi1 * e.B1 + phi2 * e.B2);
        const double AP = phi1 * e.A1 + phi2 * e.A2;
        W[0] = (float)a1r1;
        W[1] = (float)a2r2;
#pragma unroll
        for (int d = 0; d < D; ++d) W[2 + d] = (float)(U[2 + d] * ir);
        W[IE] = (float)(num * rcp_mixed(AP));  // rounded once from near-FP64: a uniform pressure stays uniform
        W[IA] = (float)alpha1;
    }

    __device__ static __forceinline__ void prim2cons(double* U, const double* W, const Eos& e, unsigned int* err) {
        const double a1r1 = W[0], a2r2 = W[1], p = W[IE], alpha1 = W[IA];
        const double rho = a1r1 + a2r2;
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = nasg_phi(alpha1, a1r1, e.C1, err);
        const double phi2 = nasg_phi(alpha2, a2r2, e.C2, err);
        const double rho_D = a1r1 * e.D1 + a2r2 * e.D2;
        const double AP = phi1 * e.A1 + phi2 * e.A2;
        const double BP = phi1 * e.B1 + phi2 * e.B2;
        const double rho_e = (AP * p + BP) + rho_D;
        U[0] = a1r1;
        U[1] = a2r2;
        for (int d = 0; d < D; ++d) U[2 + d] = rho * W[2 + d];
        U[IE] = rho_e + (0.5 * rho) * ksum<D>(W + 2);
        U[IA] = alpha1;
    }

    // THINC side of a face: the face state Uf (MUSCL-minmod) with its volume fraction replaced by the
    // THINC value af; phase densities, velocity and pressure are kept, masses, momentum and energy
    // rebuilt (Reconstruct_State_From_VolumeFraction,
    // include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible5Eq.H:15-63).
    __device__ static __forceinline__ void thinc_rebuild(double* Uo, const double* Uf, double af, const Eos& e,
                                                         unsigned int* err) {
        double W[N];
        cons2prim(W, Uf, e, err);
        const double al = W[IA], p = W[IE];
        const double rho1 = W[0] / al;
        const double rho2 = W[1] / (1.0 - al);
        const double m1 = af * rho1;
        const double m2 = (1.0 - af) * rho2;
        const double rr = m1 + m2;
        const double K = 0.5 * ksum<D>(W + 2);
        const double r1e1 = (e.C1 > 0.0) ? nasg_xi_rho(rho1, e.C1, err) * (e.A1 * p + e.B1) + rho1 * e.D1
                                         : e.A1 * p + e.B1 + rho1 * e.D1;
        const double r2e2 = (e.C2 > 0.0) ? nasg_xi_rho(rho2, e.C2, err) * (e.A2 * p + e.B2) + rho2 * e.D2
                                         : e.A2 * p + e.B2 + rho2 * e.D2;
        Uo[0] = m1;
        Uo[1] = m2;
#pragma unroll
        for (int c = 0; c < D; ++c) Uo[2 + c] = W[2 + c] * rr;
        Uo[IE] = K * rr + r1e1 * af + r2e2 * (1.0 - af);
        Uo[IA] = af;
    }

    // Mixture sound speed; source_term 0 (K = 0) or 1 (Wood).
    __device__ static __forceinline__ double sound_speed(const double* W, const Eos& e, int id_k, unsigned int* err) {
        const double a1r1 = W[0], a2r2 = W[1], p = W[IE], alpha1 = W[IA];
        const double r1c1 = ((e.A1 + 1.0) * p + e.B1) / e.A1;
        const double r2c2 = ((e.A2 + 1.0) * p + e.B2) / e.A2;
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = nasg_phi(alpha1, a1r1, e.C1, err);
        const double phi2 = nasg_phi(alpha2, a2r2, e.C2, err);
        double rho_c2;
        if (id_k == 0) {
            const double ap_rc2 = (alpha1 * e.A1) * r1c1 + (alpha2 * e.A2) * r2c2;
            const double AP = phi1 * e.A1 + phi2 * e.A2;
            rho_c2 = ap_rc2 / AP;
        } else {
            rho_c2 = 1.0 / (phi1 / r1c1 + phi2 / r2c2);
        }
        const double rho = a1r1 + a2r2;
        return sqrt(rho_c2 / rho);
    }

    // Kapila coefficient factor phi1 (1 + K1) of the alpha1 equation (FVM_SurfaceIntegralNC_Compressible5Eq.H:15-52).
    __device__ static __forceinline__ double kapila_factor(const double* U, const double* W, const Eos& e, int id_k,
                                                           unsigned int* err) {
        const double alpha1 = U[IA];
        double phi1 = (id_k == 1) ? nasg_phi(alpha1, U[0], e.C1, err) : alpha1;
        double K1 = 0.0;
        if (id_k == 1) {
            const double p = W[IE];
            const double r1c1 = ((e.A1 + 1.0) * p + e.B1) / e.A1;
            const double r2c2 = ((e.A2 + 1.0) * p + e.B2) / e.A2;
            const double alpha2 = 1.0 - alpha1;
            const double ph1 = nasg_phi(alpha1, W[0], e.C1, err);
            const double ph2 = nasg_phi(alpha2, W[1], e.C2, err);
            const double rho_c2 = 1.0 / (ph1 / r1c1 + ph2 / r2c2);
            K1 = rho_c2 / r1c1 - 1.0;
        }
        return phi1 * (1.0 + K1);
    }

    // Physical flux in direction d of the state U with primitives W (Conservative2Flux).
    __device__ static __forceinline__ void flux(double* F, const double* U, const double* W, int d) {
        const double V = pick<D>(W + 2, d);
        const double p = W[IE];
        F[0] = U[0] * V;
        F[1] = U[1] * V;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            F[2 + c] = U[2 + c] * V;
            if (c == d) F[2 + c] = F[2 + c] + p;
        }
        F[IE] = (U[IE] + p) * V;
        F[IA] = U[IA] * V;
    }

    // HLLC flux, the normal face velocity u* (FluxNC[0]) and the face wave speed, from the face
    // states UL, UR (Riemann_HLLC converts them to primitives first).
    __device__ static __forceinline__ void hllc(double* Fout, double* fnc, double& cmax, const double* UL,
                                                const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
        double WL[N], WR[N];
        cons2prim(WL, UL, e, err);
        cons2prim(WR, UR, e, err);
        hllc_uw(Fout, fnc, cmax, UL, WL, UR, WR, e, d, id_k, err);
    }

    // The same from face states given both as conserved (U) and primitive (W) variables.
    __device__ static __forceinline__ void hllc_uw(double* Fout, double* fnc, double& cmax, const double* UL,
                                                   const double* WL, const double* UR, const double* WR, const Eos& e,
                                                   int d, int id_k, unsigned int* err) {
        double FL[N], FR[N];
        flux(FL, UL, WL, d);
        flux(FR, UR, WR, d);
        const double cL = sound_speed(WL, e, id_k, err);
        const double cR = sound_speed(WR, e, id_k, err);
        const double VL = pick<D>(WL + 2, d), VR = pick<D>(WR + 2, d);
        const double pL = WL[IE], pR = WR[IE];
        const double V_avg = 0.5 * (VL + VR);
        const double c_avg = 0.5 * (cL + cR);
        const double SL = dmin(V_avg - c_avg, VL - cL);
        const double SR = dmax(V_avg + c_avg, VR + cR);
        const double Sm = dmin(0.0, SL);
        const double Sp = dmax(0.0, SR);
        const double rhoL = WL[0] + WL[1];
        const double rhoR = WR[0] + WR[1];
        const double S_Star = (((pR - pL) + (rhoL * VL) * (SL - VL)) - (rhoR * VR) * (SR - VR)) /
                              (rhoL * (SL - VL) - rhoR * (SR - VR));
        const double s = sgn0(S_Star);
        const double hp = 0.5 * (1.0 + s), hm = 0.5 * (1.0 - s);
        const double fL = (SL - VL) / (SL - S_Star);
        const double fR = (SR - VR) / (SR - S_Star);
        // normal face velocity: Vel[d] = hp*uL_d + hm*uR_d, then += hp*Sm*(fL-1) + hm*Sp*(fR-1)
        double vel = hp * VL + hm * VR;
        vel = vel + ((hp * Sm) * (fL - 1.0) + (hm * Sp) * (fR - 1.0));
        fnc[0] = vel;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double sL = fL * UL[i];
            double sR = fR * UR[i];
            if (i == 2 + d) {
                sL = sL + (fL * rhoL) * (S_Star - VL);
                sR = sR + (fR * rhoR) * (S_Star - VR);
            } else if (i == IE) {
                sL = sL + (fL * (S_Star - VL)) * (rhoL * S_Star + pL / (SL - VL));
                sR = sR + (fR * (S_Star - VR)) * (rhoR * S_Star + pR / (SR - VR));
            }
            Fout[i] = hp * (FL[i] + Sm * (sL - UL[i])) + hm * (FR[i] + Sp * (sR - UR[i]));
        }
        const double qL = cL + sqrt(ksum<D>(WL + 2));
        const double qR = cR + sqrt(ksum<D>(WR + 2));
        cmax = dmax(qL, qR);
    }
};

// Mixed-precision HLLC of the five-equation model. The wave speeds, S*, the star ratios
// f = (S - V)/(S - S*) and the divisions and square roots run in FP32 on the reconstructed face
// primitives (w); the star states and fluxes are assembled in FP64 from the FP64 face states U, so
// that the large energy (alpha B ~ 1e9) enters only through f*E and stays consistent with the
// alpha flux f*alpha (the pressure recovered from E - sum alpha_k B_k is not polluted).
// FP32 sound speeds of the mixed Riemann solvers from FP32 face primitives: five-equation mixture
// (K = 0: frozen, K = 1: Wood), six-equation frozen.
template <int DIM>
__device__ __forceinline__ float fiveeq_c_f32(const float* w, const Eos& e, int id_k) {
    using M = FiveEq<DIM>;
    constexpr int IE = M::IE, IA = M::IA;
    const float p = w[IE], a1 = w[IA], a2 = 1.0f - a1;
    const float A1 = e.fA1, A2 = e.fA2, B1 = e.fB1, B2 = e.fB2;
    const float r1 = __fdividef(__fmaf_rn(A1 + 1.0f, p, B1), A1);
    const float r2 = __fdividef(__fmaf_rn(A2 + 1.0f, p, B2), A2);
    const float ph1 = (e.fC1 > 0.0f) ? a1 - e.fC1 * w[0] : a1;
    const float ph2 = (e.fC2 > 0.0f) ? a2 - e.fC2 * w[1] : a2;
    float rc2;
    if (id_k == 0)
        rc2 = __fdividef(__fmaf_rn(a1 * A1, r1, (a2 * A2) * r2), __fmaf_rn(ph1, A1, ph2 * A2));
    else
        rc2 = __fdividef(1.0f, __fdividef(ph1, r1) + __fdividef(ph2, r2));
    return sqrtf(fmaxf(rc2, 0.0f) / (w[0] + w[1]));
}

template <int DIM>
__device__ __forceinline__ void fiveeq_hllc_mixed(double* Fout, double* fnc, float& cmax, const double* UL,
                                                  const double* UR, const float* wL, const float* wR,
                                                  const Eos& e, int d, int id_k) {
    using M = FiveEq<DIM>;
    constexpr int N = M::N, IE = M::IE, IA = M::IA;
    const float cL = fiveeq_c_f32<DIM>(wL, e, id_k), cR = fiveeq_c_f32<DIM>(wR, e, id_k);
    const float VL = (d == 0) ? wL[2] : ((d == 1 || DIM == 2) ? wL[3] : wL[DIM == 3 ? 4 : 3]);
    const float VR = (d == 0) ? wR[2] : ((d == 1 || DIM == 2) ? wR[3] : wR[DIM == 3 ? 4 : 3]);
    const float pL = wL[IE], pR = wR[IE];
    const float rhoL = wL[0] + wL[1], rhoR = wR[0] + wR[1];
    const float Va = 0.5f * (VL + VR), ca = 0.5f * (cL + cR);
    const float SL = fminf(Va - ca, VL - cL), SR = fmaxf(Va + ca, VR + cR);
    const float Sm = fminf(0.0f, SL), Sp = fmaxf(0.0f, SR);
    // delta form: dS = S* - V and f - 1 from the jumps, exactly 0 where p and V are uniform
    const float gL = SL - VL, gR = SR - VR;
    const float aL = rhoL * gL, aR = rhoR * gR;
    const float inv_den = __fdividef(1.0f, aL - aR);
    const float dp = pR - pL, dV = VL - VR;
    const float dSL = __fmaf_rn(aR, dV, dp) * inv_den, dSR = __fmaf_rn(aL, dV, dp) * inv_den;
    const float S = VL + dSL;
    const float fm1L = __fdividef(dSL, gL - dSL), fm1R = __fdividef(dSR, gR - dSR);
    const float eL = (1.0f + fm1L) * dSL * (rhoL * S + __fdividef(pL, gL));
    const float eR = (1.0f + fm1R) * dSR * (rhoR * S + __fdividef(pR, gR));
    const float mL = (1.0f + fm1L) * rhoL * dSL, mR = (1.0f + fm1R) * rhoR * dSR;
    if (S != 0.0f) {
        // FP64 assembly of the upwind side K only (left where S > 0): F = F_K + S_K (U*_K - U_K), the
        // value of the blend below, whose weights are then 1 and 0
        const bool lt = (S > 0.0f);
        const double V = lt ? VL : VR, p = lt ? pL : pR, gm = lt ? fm1L : fm1R, Sk = lt ? Sm : Sp;
        const double en = lt ? eL : eR, mo = lt ? mL : mR;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const double u = lt ? UL[i] : UR[i];
            double f = u * V, dd = gm * u;
            if (i == IE) {
                f = (u + p) * V;
                dd += en;
            } else if (i >= 2 && i < 2 + DIM && i - 2 == d) {
                f += p;
                dd += mo;
            }
            Fout[i] = fma(Sk, dd, f);
        }
        fnc[0] = fma(Sk, gm, V);
    } else {
    const float s = 0.0f;
    // FP64 assembly: F = h+ (F_L + S- (U*_L - U_L)) + h- (F_R + S+ (U*_R - U_R))
    const double hp = 0.5 * (1.0 + s), hm = 0.5 * (1.0 - s);
    const double gmL = fm1L, gmR = fm1R, Smd = Sm, Spd = Sp;
    const double VLd = VL, VRd = VR, pLd = pL, pRd = pR;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double fl = UL[i] * VLd, fr = UR[i] * VRd;
        double dL = gmL * UL[i], dR = gmR * UR[i];
        if (i == IE) {
            fl = (UL[IE] + pLd) * VLd;
            fr = (UR[IE] + pRd) * VRd;
            dL += (double)eL;
            dR += (double)eR;
        } else if (i >= 2 && i < 2 + DIM && i - 2 == d) {
            fl += pLd;
            fr += pRd;
            dL += (double)mL;
            dR += (double)mR;
        }
        Fout[i] = hp * (fl + Smd * dL) + hm * (fr + Spd * dR);
    }
    fnc[0] = (hp * VLd + hm * VRd) + ((hp * Smd) * gmL + (hm * Spd) * gmR);
    }
    float kL = wL[2] * wL[2] + wL[3] * wL[3], kR = wR[2] * wR[2] + wR[3] * wR[3];
    if (DIM == 3) { kL += wL[4] * wL[4]; kR += wR[4] * wR[4]; }
    cmax = fmaxf(cL + sqrtf(kL), cR + sqrtf(kR));
    (void)IA;
}

// ------------------------------------------------------------------------------------------------
// Six-equation model: U = (a1r1, a2r2, rho u_d, a1r1E1, a2r2E2, alpha1),
//                     W = (a1r1, a2r2, u_d, a1p1, a2p2, alpha1)
// ------------------------------------------------------------------------------------------------
template <int DIM>
struct SixEq {
    static constexpr int KIND = kModelSix;
    static constexpr int D = DIM;
    static constexpr int N = 5 + DIM;
    static constexpr int NC = 3;        // u_n, (u a1p1)_n, (u a2p2)_n
    static constexpr int NCPF = 4;      // Phase-Field step: J1 r1, J2 r2, J1 r1 EK, J2 r2 EK
    static constexpr int NP = 2;        // phases
    static constexpr int IM = 2;        // rho u_d (u_d among the primitives)
    static constexpr int IE1 = 2 + DIM;
    static constexpr int IE2 = 3 + DIM;
    static constexpr int IA = 4 + DIM;

    // alpha p of one phase from alpha rho e (EquationOfState_Phase, pressure base, e -> p)
    __device__ static __forceinline__ double phase_p(double are, double alpha, double ar, double A, double B,
                                                     double b, double Dq, unsigned int* err) {
        const double xi = nasg_xi(alpha, ar, b, err);
        const double phi = xi * alpha;
        return ((are - ar * Dq) - phi * B) / (A * xi);
    }
    // alpha rho e of one phase from alpha p (p -> e)
    __device__ static __forceinline__ double phase_e(double ap, double alpha, double ar, double A, double B,
                                                     double b, double Dq, unsigned int* err) {
        const double xi = nasg_xi(alpha, ar, b, err);
        const double phi = xi * alpha;
        return ((A * xi) * ap + phi * B) + ar * Dq;
    }

    __device__ static __forceinline__ void cons2prim(double* W, const double* U, const Eos& e, unsigned int* err) {
        const double a1r1 = U[0], a2r2 = U[1], alpha1 = U[IA];
        const double alpha2 = 1.0 - alpha1;
        const double rho = a1r1 + a2r2;
        double u[3];
        for (int d = 0; d < D; ++d) u[d] = U[2 + d] / rho;
        const double k = ksum<D>(u);
        const double a1r1e1 = U[IE1] - (0.5 * a1r1) * k;
        const double a2r2e2 = U[IE2] - (0.5 * a2r2) * k;
        W[0] = a1r1;
        W[1] = a2r2;
        for (int d = 0; d < D; ++d) W[2 + d] = u[d];
        W[IE1] = phase_p(a1r1e1, alpha1, a1r1, e.A1, e.B1, e.C1, e.D1, err);
        W[IE2] = phase_p(a2r2e2, alpha2, a2r2, e.A2, e.B2, e.C2, e.D2, err);
        W[IA] = alpha1;
    }

    // Mixed precision (see FiveEq::cons2prim_f32): phase-energy numerators in FP64, divisions in FP32.
    __device__ static __forceinline__ void cons2prim_f32(float* W, const double* U, const Eos& e) {
        const double a1r1 = U[0], a2r2 = U[1], alpha1 = U[IA];
        const double alpha2 = 1.0 - alpha1;
        const double rho = a1r1 + a2r2;
        const double ir = rcp_mixed(rho);  // near-FP64 reciprocal: u = fl32(rho u / rho) keeps uniform flow uniform
        double m2 = U[2] * U[2] + U[3] * U[3];
        if (D == 3) m2 += U[4] * U[4];
        const double k = (m2 * ir) * ir;  // |u|^2
        const float xi1 = (e.C1 > 0.0 && alpha1 > 0.0) ? (float)(1.0 - e.C1 * (a1r1 / alpha1)) : 1.0f;
        const float xi2 = (e.C2 > 0.0 && alpha2 > 0.0) ? (float)(1.0 - e.C2 * (a2r2 / alpha2)) : 1.0f;
        const double n1 = (U[IE1] - (0.5 * a1r1) * k - a1r1 * e.D1) - ((double)xi1 * alpha1) * e.B1;
        const double n2 = (U[IE2] - (0.5 * a2r2) * k - a2r2 * e.D2) - ((double)xi2 * alpha2) * e.B2;
        W[0] = (float)a1r1;
        W[1] = (float)a2r2;
#pragma unroll
        for (int d = 0; d < D; ++d) W[2 + d] = (float)(U[2 + d] * ir);
        // rounded once from FP64 (a uniform pressure stays uniform); the NASG factor 1/xi in FP32
        W[IE1] = (e.C1 > 0.0) ? (float)(n1 * e.iA1) / xi1 : (float)(n1 * e.iA1);
        W[IE2] = (e.C2 > 0.0) ? (float)(n2 * e.iA2) / xi2 : (float)(n2 * e.iA2);
        W[IA] = (float)alpha1;
    }

    __device__ static __forceinline__ void prim2cons(double* U, const double* W, const Eos& e, unsigned int* err) {
        const double a1r1 = W[0], a2r2 = W[1], alpha1 = W[IA];
        const double alpha2 = 1.0 - alpha1;
        const double rho = a1r1 + a2r2;
        U[0] = a1r1;
        U[1] = a2r2;
        for (int d = 0; d < D; ++d) U[2 + d] = rho * W[2 + d];
        const double a1r1e1 = phase_e(W[IE1], alpha1, a1r1, e.A1, e.B1, e.C1, e.D1, err);
        const double a2r2e2 = phase_e(W[IE2], alpha2, a2r2, e.A2, e.B2, e.C2, e.D2, err);
        const double k = ksum<D>(W + 2);
        U[IE1] = a1r1e1 + (0.5 * a1r1) * k;
        U[IE2] = a2r2e2 + (0.5 * a2r2) * k;
        U[IA] = alpha1;
    }

    // THINC side of a face (include/Operators_Compressible6Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible6Eq.H:14-62):
    // phase densities, velocity and phase pressures of the face state are kept.
    __device__ static __forceinline__ void thinc_rebuild(double* Uo, const double* Uf, double af, const Eos& e,
                                                         unsigned int* err) {
        double W[N];
        cons2prim(W, Uf, e, err);
        const double al = W[IA];
        const double rho1 = W[0] / al;
        const double rho2 = W[1] / (1.0 - al);
        const double m1 = af * rho1;
        const double m2 = (1.0 - af) * rho2;
        const double rr = m1 + m2;
        const double p1 = W[IE1] / al;
        const double p2 = W[IE2] / (1.0 - al);
        const double K = 0.5 * ksum<D>(W + 2);
        const double r1e1 = (e.C1 > 0.0) ? nasg_xi_rho(rho1, e.C1, err) * (e.A1 * p1 + e.B1) + rho1 * e.D1
                                         : e.A1 * p1 + e.B1 + rho1 * e.D1;
        const double r2e2 = (e.C2 > 0.0) ? nasg_xi_rho(rho2, e.C2, err) * (e.A2 * p2 + e.B2) + rho2 * e.D2
                                         : e.A2 * p2 + e.B2 + rho2 * e.D2;
        Uo[0] = m1;
        Uo[1] = m2;
#pragma unroll
        for (int c = 0; c < D; ++c) Uo[2 + c] = W[2 + c] * rr;
        Uo[IE1] = K * m1 + r1e1 * af;
        Uo[IE2] = K * m2 + r2e2 * (1.0 - af);
        Uo[IA] = af;
    }

    // Frozen mixture sound speed: rho c^2 = sum alpha_k rho_k c_k^2.
    __device__ static __forceinline__ double sound_speed(const double* W, const Eos& e, unsigned int* err) {
        const double a1r1 = W[0], a2r2 = W[1], alpha1 = W[IA];
        const double xi1 = nasg_xi(alpha1, a1r1, e.C1, err);
        const double xi2 = nasg_xi(1.0 - alpha1, a2r2, e.C2, err);
        const double r1c1 = ((e.A1 + 1.0) * W[IE1] + alpha1 * e.B1) / (e.A1 * xi1);
        const double r2c2 = ((e.A2 + 1.0) * W[IE2] + (1.0 - alpha1) * e.B2) / (e.A2 * xi2);
        const double rho_c2 = r1c1 + r2c2;
        const double rho = a1r1 + a2r2;
        return sqrt(rho_c2 / rho);
    }

    __device__ static __forceinline__ void flux(double* F, const double* U, const double* W, int d) {
        const double V = pick<D>(W + 2, d);
        F[0] = U[0] * V;
        F[1] = U[1] * V;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            F[2 + c] = U[2 + c] * V;
            if (c == d) F[2 + c] = F[2 + c] + (W[IE1] + W[IE2]);
        }
        F[IE1] = (U[IE1] + W[IE1]) * V;
        F[IE2] = (U[IE2] + W[IE2]) * V;
        F[IA] = U[IA] * V;
    }

    // HLLC flux and the face quantities u_n, (u a1p1)_n, (u a2p2)_n of the non-conservative terms.
    __device__ static __forceinline__ void hllc(double* Fout, double* fnc, double& cmax, const double* UL,
                                                const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
        double WL[N], WR[N];
        cons2prim(WL, UL, e, err);
        cons2prim(WR, UR, e, err);
        hllc_uw(Fout, fnc, cmax, UL, WL, UR, WR, e, d, id_k, err);
    }

    __device__ static __forceinline__ void hllc_uw(double* Fout, double* fnc, double& cmax, const double* UL,
                                                   const double* WL, const double* UR, const double* WR, const Eos& e,
                                                   int d, int /*id_k*/, unsigned int* err) {
        double FL[N], FR[N];
        flux(FL, UL, WL, d);
        flux(FR, UR, WR, d);
        const double cL = sound_speed(WL, e, err);
        const double cR = sound_speed(WR, e, err);
        const double VL = pick<D>(WL + 2, d), VR = pick<D>(WR + 2, d);
        const double SL = dmin(VL - cL, VR - cR);
        const double SR = dmax(VL + cL, VR + cR);
        const double Sm = dmin(0.0, SL);
        const double Sp = dmax(0.0, SR);
        const double a1r1L = WL[0], a2r2L = WL[1], a1r1R = WR[0], a2r2R = WR[1];
        const double a1p1L = WL[IE1], a2p2L = WL[IE2], a1p1R = WR[IE1], a2p2R = WR[IE2];
        const double rhoL = a1r1L + a2r2L;
        const double rhoR = a1r1R + a2r2R;
        const double pL = a1p1L + a2p2L;
        const double pR = a1p1R + a2p2R;
        const double S_Star = (((pR - pL) + (rhoL * VL) * (SL - VL)) - (rhoR * VR) * (SR - VR)) /
                              (rhoL * (SL - VL) - rhoR * (SR - VR));
        const double fL = (SL - VL) / (SL - S_Star);
        const double fR = (SR - VR) / (SR - S_Star);
        const double a1r1Ls = fL * a1r1L, a1r1Rs = fR * a1r1R;
        const double a2r2Ls = fL * a2r2L, a2r2Rs = fR * a2r2R;
        double UsL[N], UsR[N];
        UsL[0] = a1r1Ls; UsL[1] = a2r2Ls;
        UsR[0] = a1r1Rs; UsR[1] = a2r2Rs;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double uLc = WL[2 + c], uRc = WR[2 + c];
            const double nrm = (c == d) ? 1.0 : 0.0;
            UsL[2 + c] = (fL * rhoL) * (uLc + nrm * (S_Star - uLc));
            UsR[2 + c] = (fR * rhoR) * (uRc + nrm * (S_Star - uRc));
        }
        const double a1p1Ls = (a1p1L + ((VL - SL) * a1r1L) * VL) - ((S_Star - SL) * a1r1Ls) * S_Star;
        const double a1p1Rs = (a1p1R + ((VR - SR) * a1r1R) * VR) - ((S_Star - SR) * a1r1Rs) * S_Star;
        const double a2p2Ls = (a2p2L + ((VL - SL) * a2r2L) * VL) - ((S_Star - SL) * a2r2Ls) * S_Star;
        const double a2p2Rs = (a2p2R + ((VR - SR) * a2r2R) * VR) - ((S_Star - SR) * a2r2Rs) * S_Star;
        UsL[IE1] = (((VL - SL) * UL[IE1] + VL * a1p1L) - S_Star * a1p1Ls) / (S_Star - SL);
        UsR[IE1] = (((VR - SR) * UR[IE1] + VR * a1p1R) - S_Star * a1p1Rs) / (S_Star - SR);
        UsL[IE2] = (((VL - SL) * UL[IE2] + VL * a2p2L) - S_Star * a2p2Ls) / (S_Star - SL);
        UsR[IE2] = (((VR - SR) * UR[IE2] + VR * a2p2R) - S_Star * a2p2Rs) / (S_Star - SR);
        UsL[IA] = fL * WL[IA];
        UsR[IA] = fR * WR[IA];
        const double s = sgn0(S_Star);
        const double hp = 0.5 * (1.0 + s), hm = 0.5 * (1.0 - s);
        // normal components of Vel, Vel*a1p1, Vel*a2p2
        const double uLd = VL, uRd = VR;
        double vel = hp * uLd + hm * uRd;
        vel = vel + ((hp * Sm) * (fL - 1.0) + (hm * Sp) * (fR - 1.0));
        const double va1 = hp * (uLd * a1p1L + (1.0 * Sm) * (VL * a1p1L - S_Star * a1p1Ls) / (S_Star - SL)) +
                           hm * (uRd * a1p1R + (1.0 * Sp) * (VR * a1p1R - S_Star * a1p1Rs) / (S_Star - SR));
        const double va2 = hp * (uLd * a2p2L + (1.0 * Sm) * (VL * a2p2L - S_Star * a2p2Ls) / (S_Star - SL)) +
                           hm * (uRd * a2p2R + (1.0 * Sp) * (VR * a2p2R - S_Star * a2p2Rs) / (S_Star - SR));
        fnc[0] = vel;
        fnc[1] = va1;
        fnc[2] = va2;
#pragma unroll
        for (int i = 0; i < N; ++i)
            Fout[i] = hp * (FL[i] + Sm * (UsL[i] - UL[i])) + hm * (FR[i] + Sp * (UsR[i] - UR[i]));
        const double qL = cL + sqrt(ksum<D>(WL + 2));
        const double qR = cR + sqrt(ksum<D>(WR + 2));
        cmax = dmax(qL, qR);
    }
};

// Mixed-precision HLLC of the six-equation model (same split as fiveeq_hllc_mixed). The phase-energy
// star states are written E* = f E + (V alpha p - S* (alpha p)*)/(S* - S), the identity of
// Riemann_HLLC_Compressible6Eq.H:163-200 with (V - S)/(S* - S) = f, so that E enters only through f.
template <int DIM>
__device__ __forceinline__ float sixeq_c_f32(const float* w, const Eos& e) {
    using M = SixEq<DIM>;
    constexpr int IE1 = M::IE1, IE2 = M::IE2, IA = M::IA;
    const float a1 = w[IA];
    const float xi1 = (e.fC1 > 0.0f && a1 > 0.0f) ? 1.0f - e.fC1 * __fdividef(w[0], a1) : 1.0f;
    const float xi2 = (e.fC2 > 0.0f && 1.0f - a1 > 0.0f) ? 1.0f - e.fC2 * __fdividef(w[1], 1.0f - a1) : 1.0f;
    const float r1 = __fdividef(__fmaf_rn(e.fA1 + 1.0f, w[IE1], a1 * e.fB1), e.fA1 * xi1);
    const float r2 = __fdividef(__fmaf_rn(e.fA2 + 1.0f, w[IE2], (1.0f - a1) * e.fB2), e.fA2 * xi2);
    return sqrtf(fmaxf(r1 + r2, 0.0f) / (w[0] + w[1]));
}

template <int DIM>
__device__ __forceinline__ void sixeq_hllc_mixed(double* Fout, double* fnc, float& cmax, const double* UL,
                                                 const double* UR, const float* wL, const float* wR,
                                                 const Eos& e, int d) {
    using M = SixEq<DIM>;
    constexpr int N = M::N, IE1 = M::IE1, IE2 = M::IE2, IA = M::IA;
    const float cL = sixeq_c_f32<DIM>(wL, e), cR = sixeq_c_f32<DIM>(wR, e);
    const float VL = (d == 0) ? wL[2] : ((d == 1 || DIM == 2) ? wL[3] : wL[DIM == 3 ? 4 : 3]);
    const float VR = (d == 0) ? wR[2] : ((d == 1 || DIM == 2) ? wR[3] : wR[DIM == 3 ? 4 : 3]);
    const float SL = fminf(VL - cL, VR - cR), SR = fmaxf(VL + cL, VR + cR);
    const float Sm = fminf(0.0f, SL), Sp = fmaxf(0.0f, SR);
    const float rhoL = wL[0] + wL[1], rhoR = wR[0] + wR[1];
    const float pL = wL[IE1] + wL[IE2], pR = wR[IE1] + wR[IE2];
    // delta form: dS = S* - V and f - 1 from the jumps, exactly 0 where p and V are uniform
    const float gL = SL - VL, gR = SR - VR;
    const float aL = rhoL * gL, aR = rhoR * gR;
    const float inv_den = __fdividef(1.0f, aL - aR);
    const float dp = pR - pL, dV = VL - VR;
    const float dSL = __fmaf_rn(aR, dV, dp) * inv_den, dSR = __fmaf_rn(aL, dV, dp) * inv_den;
    const float S = VL + dSL;
    const float qL = __fdividef(dSL, gL - dSL), qR = __fdividef(dSR, gR - dSR);  // f - 1
    const float fL = 1.0f + qL, fR = 1.0f + qR;
    // phase pressures at the star state: (alpha p)* = alpha p + alpha rho (S - V) dS, and the
    // pressure part t of the phase-energy star state E* = f E + t, t = dS ((alpha p) + S* alpha rho g)/(g - dS)
    const float a1p1L = wL[IE1], a2p2L = wL[IE2], a1p1R = wR[IE1], a2p2R = wR[IE2];
    const float tL1 = qL * __fmaf_rn(S * wL[0], gL, a1p1L), tR1 = qR * __fmaf_rn(S * wR[0], gR, a1p1R);
    const float tL2 = qL * __fmaf_rn(S * wL[1], gL, a2p2L), tR2 = qR * __fmaf_rn(S * wR[1], gR, a2p2R);
    const float mL = fL * rhoL * dSL, mR = fR * rhoR * dSR;
    if (S != 0.0f) {
        // FP64 assembly of the upwind side K only (left where S > 0): F = F_K + S_K (U*_K - U_K), the
        // value of the blend below, whose weights are then 1 and 0
        const bool lt = (S > 0.0f);
        const double V = lt ? VL : VR, gm = lt ? qL : qR, Sk = lt ? Sm : Sp;
        const double p1 = lt ? a1p1L : a1p1R, p2 = lt ? a2p2L : a2p2R;
        const double mo = lt ? mL : mR, t1 = lt ? tL1 : tR1, t2 = lt ? tL2 : tR2;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const double u = lt ? UL[i] : UR[i];
            double f = u * V, dd = gm * u;
            if (i >= 2 && i < 2 + DIM && i - 2 == d) {
                f += p1 + p2;
                dd += mo;
            } else if (i == IE1) {
                f = (u + p1) * V;
                dd += t1;
            } else if (i == IE2) {
                f = (u + p2) * V;
                dd += t2;
            }
            Fout[i] = fma(Sk, dd, f);
        }
        fnc[0] = fma(Sk, gm, V);
        fnc[1] = fma(Sk, t1, V * p1);
        fnc[2] = fma(Sk, t2, V * p2);
    } else {
    const float s = 0.0f;
    const double hp = 0.5 * (1.0 + s), hm = 0.5 * (1.0 - s);
    const double gmL = qL, gmR = qR, Smd = Sm, Spd = Sp;
    const double VLd = VL, VRd = VR;
    const double p1L = a1p1L, p2L = a2p2L, p1R = a1p1R, p2R = a2p2R;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double fl = UL[i] * VLd, fr = UR[i] * VRd;
        double dL = gmL * UL[i], dR = gmR * UR[i];
        if (i >= 2 && i < 2 + DIM && i - 2 == d) {
            fl += p1L + p2L;
            fr += p1R + p2R;
            dL += (double)mL;
            dR += (double)mR;
        } else if (i == IE1) {
            fl = (UL[IE1] + p1L) * VLd;
            fr = (UR[IE1] + p1R) * VRd;
            dL += (double)tL1;
            dR += (double)tR1;
        } else if (i == IE2) {
            fl = (UL[IE2] + p2L) * VLd;
            fr = (UR[IE2] + p2R) * VRd;
            dL += (double)tL2;
            dR += (double)tR2;
        }
        Fout[i] = hp * (fl + Smd * dL) + hm * (fr + Spd * dR);
    }
    fnc[0] = (hp * VLd + hm * VRd) + ((hp * Smd) * gmL + (hm * Spd) * gmR);
    fnc[1] = hp * (VLd * p1L + Smd * (double)tL1) + hm * (VRd * p1R + Spd * (double)tR1);
    fnc[2] = hp * (VLd * p2L + Smd * (double)tL2) + hm * (VRd * p2R + Spd * (double)tR2);
    }
    float kL = wL[2] * wL[2] + wL[3] * wL[3], kR = wR[2] * wR[2] + wR[3] * wR[3];
    if (DIM == 3) { kL += wL[4] * wL[4]; kR += wR[4] * wR[4]; }
    cmax = fmaxf(cL + sqrtf(kL), cR + sqrtf(kR));
}

// ------------------------------------------------------------------------------------------------
// WENO5 face value, epsilon-free weights from smoothness ratios with a NaN guard.
// side = +1: value at the right face of the centre cell c; side = -1: at its left face.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double weno5(double f_mm, double f_m, double f_c, double f_p, double f_pp, int side) {
    double q0, q1, q2, d0, d2;
    if (side == 1) {
        q0 = (f_c + (2.0 / 3.0) * (f_p - f_c)) - (1.0 / 6.0) * (f_pp - f_p);
        q1 = (f_c + (1.0 / 6.0) * (f_c - f_m)) + (1.0 / 3.0) * (f_p - f_c);
        q2 = (f_c - (1.0 / 3.0) * (f_m - f_mm)) + (5.0 / 6.0) * (f_c - f_m);
        d0 = 3.0 / 10.0;
        d2 = 1.0 / 10.0;
    } else {
        q0 = (f_c - (5.0 / 6.0) * (f_p - f_c)) + (1.0 / 3.0) * (f_pp - f_p);
        q1 = (f_c - (1.0 / 3.0) * (f_c - f_m)) - (1.0 / 6.0) * (f_p - f_c);
        q2 = (f_c + (1.0 / 6.0) * (f_m - f_mm)) - (2.0 / 3.0) * (f_c - f_m);
        d0 = 1.0 / 10.0;
        d2 = 3.0 / 10.0;
    }
    const double d1 = (1.0 - d0) - d2;
    const double a = f_p - f_c, b = f_pp - f_p, c = f_c - f_m, g = f_m - f_mm;
    const double IS0 = ((10.0 / 3.0) * a) * a - ((11.0 / 3.0) * a) * b + ((4.0 / 3.0) * b) * b;
    const double IS1 = (-(5.0 / 3.0) * c) * a + ((4.0 / 3.0) * c) * c + ((4.0 / 3.0) * a) * a;
    const double IS2 = ((10.0 / 3.0) * c) * c - ((11.0 / 3.0) * g) * c + ((4.0 / 3.0) * g) * g;
    double IS01 = IS0 / IS1;
    if (isnan(IS01)) IS01 = 1.0;
    const double IS10 = 1.0 / IS01;
    double IS02 = IS0 / IS2;
    if (isnan(IS02)) IS02 = 1.0;
    const double IS20 = 1.0 / IS02;
    double IS12 = IS1 / IS2;
    if (isnan(IS12)) IS12 = 1.0;
    const double IS21 = 1.0 / IS12;
    const double w0 = d0 / ((d0 + (IS01 * IS01) * d1) + (IS02 * IS02) * d2);
    const double w1 = d1 / (((IS10 * IS10) * d0 + d1) + (IS12 * IS12) * d2);
    const double w2 = d2 / (((IS20 * IS20) * d0 + (IS21 * IS21) * d1) + d2);
    double f = 0.0;
    f += w0 * q0;
    f += w1 * q1;
    f += w2 * q2;
    return f;
}

// WENO5 candidate values q and nonlinear weights w separately (WENO5.H:12-75), for the bounded
// variant, which reconstructs the volume fractions with the weights of the partial densities.
__device__ __forceinline__ void weno5_parts(double f_mm, double f_m, double f_c, double f_p, double f_pp, int side,
                                            double q[3], double* w) {
    double d0, d2;
    if (side == 1) {
        q[0] = (f_c + (2.0 / 3.0) * (f_p - f_c)) - (1.0 / 6.0) * (f_pp - f_p);
        q[1] = (f_c + (1.0 / 6.0) * (f_c - f_m)) + (1.0 / 3.0) * (f_p - f_c);
        q[2] = (f_c - (1.0 / 3.0) * (f_m - f_mm)) + (5.0 / 6.0) * (f_c - f_m);
        d0 = 3.0 / 10.0;
        d2 = 1.0 / 10.0;
    } else {
        q[0] = (f_c - (5.0 / 6.0) * (f_p - f_c)) + (1.0 / 3.0) * (f_pp - f_p);
        q[1] = (f_c - (1.0 / 3.0) * (f_c - f_m)) - (1.0 / 6.0) * (f_p - f_c);
        q[2] = (f_c + (1.0 / 6.0) * (f_m - f_mm)) - (2.0 / 3.0) * (f_c - f_m);
        d0 = 1.0 / 10.0;
        d2 = 3.0 / 10.0;
    }
    if (!w) return;
    const double d1 = (1.0 - d0) - d2;
    const double a = f_p - f_c, b = f_pp - f_p, c = f_c - f_m, g = f_m - f_mm;
    const double IS0 = ((10.0 / 3.0) * a) * a - ((11.0 / 3.0) * a) * b + ((4.0 / 3.0) * b) * b;
    const double IS1 = (-(5.0 / 3.0) * c) * a + ((4.0 / 3.0) * c) * c + ((4.0 / 3.0) * a) * a;
    const double IS2 = ((10.0 / 3.0) * c) * c - ((11.0 / 3.0) * g) * c + ((4.0 / 3.0) * g) * g;
    double IS01 = IS0 / IS1;
    if (isnan(IS01)) IS01 = 1.0;
    const double IS10 = 1.0 / IS01;
    double IS02 = IS0 / IS2;
    if (isnan(IS02)) IS02 = 1.0;
    const double IS20 = 1.0 / IS02;
    double IS12 = IS1 / IS2;
    if (isnan(IS12)) IS12 = 1.0;
    const double IS21 = 1.0 / IS12;
    w[0] = d0 / ((d0 + (IS01 * IS01) * d1) + (IS02 * IS02) * d2);
    w[1] = d1 / (((IS10 * IS10) * d0 + d1) + (IS12 * IS12) * d2);
    w[2] = d2 / (((IS20 * IS20) * d0 + (IS21 * IS21) * d1) + d2);
}

__device__ __forceinline__ double weno_sum(const double q[3], const double w[3]) {
    double f = 0.0;
    f += w[0] * q[0];
    f += w[1] * q[1];
    f += w[2] * q[2];
    return f;
}

// Positivity limiter of a cell with face values fL (right face) and fR (left face), lower bound 0
// (Limiter_Bound with ID_BoundType = -1: Limiter_BoundMin.H, fC_QuadratureRule.H; quadrature weight W:
// 1/12 for the fifth-order polynomial, 1/6 for the third-order one, FiniteVolume_Parameter.H:157-170).
__device__ __forceinline__ double bound_min_theta(double f_c, double fL, double fR, double W = 1.0 / 12.0) {
    const double fC = ((f_c - W * fL) - W * fR) / (1.0 - 2.0 * W);
    double mn = fC;  // std::min({fC, fL, fR})
    if (fL < mn) mn = fL;
    if (fR < mn) mn = fR;
    const double th = dmax(0.0, f_c - 0.0) / dmax(0.0, f_c - mn);
    return dmin(1.0, th);
}

// Bounded WENO5 (WENO5B) face values of the masses and volume fractions of one cell (stencil values
// ar1[5], ar2[5], al1[5] centred at index 2): positivity of alpha_k rho_k, alpha_k with consistent
// weights, renormalisation of sum alpha_k = 1, a second limiting pass; returns the values at the
// face `side` (+1 right, -1 left). include/Operators_Compressible5Eq/
// FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq.H:15-320 and the six-equation
// counterpart (same steps).
// Both faces of the cell: the right-face values to Wp[0], Wp[1], Wp[ia], the left-face values to
// Wm[0], Wm[1], Wm[ia]; W the quadrature weight of the positivity limiter (1/12 for WENO5B, 1/6 where
// the bound-preserving path runs it for a third-order scheme, FiniteVolume_Parameter.H:60-173).
__device__ __forceinline__ void weno5b_masses_both(const double* ar1, const double* ar2, const double* al1, double W,
                                                   double* Wp, double* Wm, int ia) {
    double rL[2], rR[2], aL[2], aR[2];
    double sumL = 0.0, sumR = 0.0;
    double ac[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double* fr = (k == 0) ? ar1 : ar2;
        double fa[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) fa[s] = (k == 0) ? al1[s] : 1.0 - al1[s];
        ac[k] = fa[2];
        double q[3], w[3], qa[3];
        weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], 1, q, w);
        rL[k] = weno_sum(q, w);
        weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], 1, qa, nullptr);
        aL[k] = weno_sum(qa, w);
        weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], -1, q, w);
        rR[k] = weno_sum(q, w);
        weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], -1, qa, nullptr);
        aR[k] = weno_sum(qa, w);
        const double th_r = bound_min_theta(fr[2], rL[k], rR[k], W);
        const double th_a = bound_min_theta(fa[2], aL[k], aR[k], W);
        const double th = dmin(th_r, th_a);
        rL[k] = fr[2] + th * (rL[k] - fr[2]);
        aL[k] = fa[2] + th * (aL[k] - fa[2]);
        rR[k] = fr[2] + th * (rR[k] - fr[2]);
        aR[k] = fa[2] + th * (aR[k] - fa[2]);
        sumL += aL[k];
        sumR += aR[k];
    }
    double Th = 1.0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double rc = (k == 0) ? ar1[2] : ar2[2];
        rL[k] /= sumL;
        aL[k] /= sumL;
        rR[k] /= sumR;
        aR[k] /= sumR;
        const double th_r = bound_min_theta(rc, rL[k], rR[k], W);
        const double th_a = bound_min_theta(ac[k], aL[k], aR[k], W);
        if (th_r < Th) Th = th_r;  // std::min({Th, th_r, th_a})
        if (th_a < Th) Th = th_a;
    }
    Wp[0] = ar1[2] + Th * (rL[0] - ar1[2]);
    Wp[1] = ar2[2] + Th * (rL[1] - ar2[2]);
    Wp[ia] = al1[2] + Th * (aL[0] - al1[2]);
    Wm[0] = ar1[2] + Th * (rR[0] - ar1[2]);
    Wm[1] = ar2[2] + Th * (rR[1] - ar2[2]);
    Wm[ia] = al1[2] + Th * (aR[0] - al1[2]);
}

__device__ __forceinline__ void weno5b_masses(const double* ar1, const double* ar2, const double* al1, int side,
                                              double& a1r1_f, double& a2r2_f, double& alpha1_f) {
    double Wp[3], Wm[3];
    weno5b_masses_both(ar1, ar2, al1, 1.0 / 12.0, Wp, Wm, 2);
    const double* Wf = (side == 1) ? Wp : Wm;
    a1r1_f = Wf[0];
    a2r2_f = Wf[1];
    alpha1_f = Wf[2];
}

// ------------------------------------------------------------------------------------------------
// Mixed precision: WENO5 / WENO5B in FP32 on primitive variables.
//
// The face value is formed as f_c + sum_k w_k (q_k - f_c), with the candidate corrections q_k - f_c
// built from the undivided differences, so a constant field is reconstructed exactly whatever the
// rounding of the weights, and the FP32 error scales with the correction, not with |f|. The
// weights are the reference's ratio-form weights (include/Operators_FV/WENO5.H:44-75) rewritten
// with one reciprocal: with r01 = IS0/IS1 and r02 = IS0/IS2, D = d0 + r01^2 d1 + r02^2 d2 and
// w0 = d0/D, w1 = d1 r01^2/D, w2 = d2 r02^2/D (the same weights in exact arithmetic); where a
// smoothness indicator vanishes or a ratio is huge, the ratio form with its NaN guard is used.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void weno5_f32_parts(float f_mm, float f_m, float f_c, float f_p, float f_pp, int side,
                                                float e[3], float* w) {
    const float a = f_p - f_c, b = f_pp - f_p, c = f_c - f_m, g = f_m - f_mm;
    float d0, d2;
    if (side == 1) {
        e[0] = __fmaf_rn(2.0f / 3.0f, a, -(1.0f / 6.0f) * b);
        e[1] = __fmaf_rn(1.0f / 6.0f, c, (1.0f / 3.0f) * a);
        e[2] = __fmaf_rn(-(1.0f / 3.0f), g, (5.0f / 6.0f) * c);
        d0 = 0.3f;
        d2 = 0.1f;
    } else {
        e[0] = __fmaf_rn(-(5.0f / 6.0f), a, (1.0f / 3.0f) * b);
        e[1] = __fmaf_rn(-(1.0f / 3.0f), c, -(1.0f / 6.0f) * a);
        e[2] = __fmaf_rn(1.0f / 6.0f, g, -(2.0f / 3.0f) * c);
        d0 = 0.1f;
        d2 = 0.3f;
    }
    if (!w) return;
    const float d1 = 0.6f;
    const float IS0 = __fmaf_rn((10.0f / 3.0f) * a, a, __fmaf_rn(-(11.0f / 3.0f) * a, b, (4.0f / 3.0f) * b * b));
    const float IS1 = __fmaf_rn(-(5.0f / 3.0f) * c, a, (4.0f / 3.0f) * __fmaf_rn(c, c, a * a));
    const float IS2 = __fmaf_rn((10.0f / 3.0f) * c, c, __fmaf_rn(-(11.0f / 3.0f) * g, c, (4.0f / 3.0f) * g * g));
    // Where some indicators vanish the ratio form gives the stencils with IS = 0 the weight in
    // proportion to their linear weights and the others none (a uniform stencil: d_k); otherwise the
    // one-reciprocal form, with the ratios clamped at 1e18 where the weights are 0 or 1 to FP32
    // precision anyway. Both are evaluated without branches.
    const bool z0 = (IS0 == 0.0f), z1 = (IS1 == 0.0f), z2 = (IS2 == 0.0f);
    const bool anyz = z0 | z1 | z2;
    const float szero = (z0 ? d0 : 0.0f) + (z1 ? d1 : 0.0f) + (z2 ? d2 : 0.0f);
    // |ratio|: an indicator can round slightly below zero; the clamp then also bounds the square
    const float r01 = fminf(fabsf(IS0 * __fdividef(1.0f, IS1)), 1.0e18f);
    const float r02 = fminf(fabsf(IS0 * __fdividef(1.0f, IS2)), 1.0e18f);
    const float s01 = anyz ? 0.0f : r01 * r01, s02 = anyz ? 0.0f : r02 * r02;
    const float den = anyz ? szero : __fmaf_rn(s01, d1, __fmaf_rn(s02, d2, d0));
    const float inv = __fdividef(1.0f, den);
    w[0] = (anyz ? (z0 ? d0 : 0.0f) : d0) * inv;
    w[1] = (anyz ? (z1 ? d1 : 0.0f) : d1 * s01) * inv;
    w[2] = (anyz ? (z2 ? d2 : 0.0f) : d2 * s02) * inv;
}

__device__ __forceinline__ float weno5_f32(float f_mm, float f_m, float f_c, float f_p, float f_pp, int side) {
    float e[3], w[3];
    weno5_f32_parts(f_mm, f_m, f_c, f_p, f_pp, side, e, w);
    return f_c + __fmaf_rn(w[0], e[0], __fmaf_rn(w[1], e[1], w[2] * e[2]));
}

// ------------------------------------------------------------------------------------------------
// GODUNOV and MUSCL face values (FiniteVolume.Scheme = GODUNOV, MUSCL-Minmod / -vanLeer / -Superbee /
// -MC; ID_Limiter 0..4), in primitive variables like WENO5:
//   include/Operators_FV/Reconstruction2Face_MUSCL_D.H (slopes (f_c - f_m)/dx, (f_p - f_m)/(2 dx),
//   (f_p - f_c)/dx), Slope_TVD.H, Limiter_Minmod.H, Limiter_vanLeer.H, Limiter_Superbee.H,
//   Limiter_MC.H, Reconstruction2Face_Linear.H (f_c + side 0.5 slope dx), Reconstruction2Face_Godunov_D.H
//   (f_c), include/Tools/Sign.H. std::min / std::max over a list keep the first extremum, as the folds
//   of dmin / dmax below do.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double sign3(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

__device__ __forceinline__ double tvd_slope(double sm, double sc, double sp, int lim) {
    if (lim == 1) return dmin(dmax(sm, 0.0), dmax(sp, 0.0)) + dmax(dmin(sm, 0.0), dmin(sp, 0.0));
    if (lim == 2) return (sm * sp > 0.0) ? 2.0 / (1.0 / sm + 1.0 / sp) : 0.0;
    if (lim == 3) {
        const double am = fabs(sm), ap = fabs(sp);
        return (sign3(sm) + sign3(sp)) * dmin(dmin(am, ap), 0.5 * dmax(am, ap));
    }
    // lim == 4: MC(a = sm, b = sp, c = sc)
    return dmin(dmin(dmax(sc, 0.0), dmax(2.0 * sm, 0.0)), dmax(2.0 * sp, 0.0)) +
           dmax(dmax(dmin(sc, 0.0), dmin(2.0 * sm, 0.0)), dmin(2.0 * sp, 0.0));
}

// Face value of the centre cell f_c on its side `side` (+1 right face, -1 left face).
__device__ __forceinline__ double muscl_face(double f_m, double f_c, double f_p, double dx, int side, int lim) {
    if (lim == 0) return f_c;
    const double s_m = (f_c - f_m) / dx;
    const double s_c = (f_p - f_m) / (2.0 * dx);
    const double s_p = (f_p - f_c) / dx;
    const double s = tvd_slope(s_m, s_c, s_p, lim);
    return f_c + (double)side * 0.5 * s * dx;
}

// WENO3 face value (FiniteVolume.Scheme = WENO3: include/Operators_FV/WENO3.H, Reconstruction2Face_WENO3_D.H,
// Reconstruction2Face_WENO.H): two candidates, ratio-form weights with the NaN guard, the weighted sum
// accumulated from 0.
__device__ __forceinline__ void weno3_qw(double f_m, double f_c, double f_p, int side, double q[2], double w[2]) {
    double q0, q1, d0;
    if (side == 1) {
        q0 = f_c + 0.5 * (f_c - f_m);
        q1 = f_c + 0.5 * (f_p - f_c);
        d0 = 1.0 / 3.0;
    } else {
        q0 = f_c - 0.5 * (f_c - f_m);
        q1 = f_c - 0.5 * (f_p - f_c);
        d0 = 2.0 / 3.0;
    }
    const double d1 = 1.0 - d0;
    const double IS0 = (f_c - f_m) * (f_c - f_m);
    const double IS1 = (f_p - f_c) * (f_p - f_c);
    double IS01 = IS0 / IS1;
    if (isnan(IS01)) IS01 = 1.0;
    const double IS10 = 1.0 / IS01;
    q[0] = q0;
    q[1] = q1;
    w[0] = d0 / (d0 + (IS01 * IS01) * d1);
    w[1] = d1 / ((IS10 * IS10) * d0 + d1);
}

__device__ __forceinline__ double weno3_sum(const double q[2], const double w[2]) {
    double f = 0.0;
    f += w[0] * q[0];
    f += w[1] * q[1];
    return f;
}

__device__ __forceinline__ double weno3_face(double f_m, double f_c, double f_p, int side) {
    double q[2], w[2];
    weno3_qw(f_m, f_c, f_p, side, q, w);
    return weno3_sum(q, w);
}

// Three-cell face values of the stage kernel's SCHEME 2: code 0..4 the GODUNOV / MUSCL family, 10 WENO3,
// 11 WENO3B (WENO3 here; the masses and volume fractions are bounded afterwards).
__device__ __forceinline__ double face3(double f_m, double f_c, double f_p, double dx, int side, int code) {
    return (code >= 10) ? weno3_face(f_m, f_c, f_p, side) : muscl_face(f_m, f_c, f_p, dx, side, code);
}

// Mixed precision: the limiters are homogeneous of degree one in the slopes, so the FP32 form limits
// the undivided differences and adds half the limited difference.
__device__ __forceinline__ float tvd_slope_f32(float sm, float sc, float sp, int lim) {
    if (lim == 1) return fminf(fmaxf(sm, 0.0f), fmaxf(sp, 0.0f)) + fmaxf(fminf(sm, 0.0f), fminf(sp, 0.0f));
    if (lim == 2) return (sm * sp > 0.0f) ? 2.0f * sm * sp / (sm + sp) : 0.0f;
    if (lim == 3) {
        const float am = fabsf(sm), ap = fabsf(sp);
        const float sg = ((sm > 0.0f) ? 1.0f : ((sm < 0.0f) ? -1.0f : 0.0f)) + ((sp > 0.0f) ? 1.0f : ((sp < 0.0f) ? -1.0f : 0.0f));
        return sg * fminf(fminf(am, ap), 0.5f * fmaxf(am, ap));
    }
    return fminf(fminf(fmaxf(sc, 0.0f), fmaxf(2.0f * sm, 0.0f)), fmaxf(2.0f * sp, 0.0f)) +
           fmaxf(fmaxf(fminf(sc, 0.0f), fminf(2.0f * sm, 0.0f)), fminf(2.0f * sp, 0.0f));
}

__device__ __forceinline__ float muscl_face_f32(float f_m, float f_c, float f_p, int side, int lim) {
    if (lim == 0) return f_c;
    const float s = tvd_slope_f32(f_c - f_m, 0.5f * (f_p - f_m), f_p - f_c, lim);
    return __fmaf_rn((float)side * 0.5f, s, f_c);
}

// WENO3 in FP32 in the correction form of weno5_f32 (f_c plus the weighted corrections), the weights
// from the ratio of the indicators with one reciprocal.
// Weight of the left candidate from the undivided differences a = f_c - f_m, b = f_p - f_c.
__device__ __forceinline__ float weno3_w0_f32(float a, float b, int side) {
    const float d0 = (side == 1) ? (1.0f / 3.0f) : (2.0f / 3.0f), d1 = 1.0f - d0;
    const float IS0 = a * a, IS1 = b * b;
    float w0;
    if (IS0 == 0.0f && IS1 == 0.0f) w0 = d0;
    else if (IS1 == 0.0f) w0 = 0.0f;
    else {
        const float r = fminf(IS0 / IS1, 1.0e18f);
        w0 = d0 / __fmaf_rn(r * r, d1, d0);
    }
    return w0;
}

__device__ __forceinline__ float weno3_face_f32(float f_m, float f_c, float f_p, int side) {
    const float a = f_c - f_m, b = f_p - f_c;
    const float h = (side == 1) ? 0.5f : -0.5f;
    return f_c + h * __fmaf_rn(weno3_w0_f32(a, b, side), a - b, b);
}

__device__ __forceinline__ float face3_f32(float f_m, float f_c, float f_p, int side, int code) {
    return (code >= 10) ? weno3_face_f32(f_m, f_c, f_p, side) : muscl_face_f32(f_m, f_c, f_p, side, code);
}

__device__ __forceinline__ float bound_min_theta_f32(float f_c, float fL, float fR, float W = 1.0f / 12.0f) {
    const float fC = (f_c - W * fL - W * fR) * (1.0f / (1.0f - 2.0f * W));
    float mn = fminf(fC, fminf(fL, fR));
    const float den = f_c - mn;
    if (!(den > 0.0f)) return 1.0f;
    return fminf(1.0f, __fdividef(fmaxf(0.0f, f_c), den));
}

// WENO5B masses and volume fraction in FP32 (same steps as weno5b_masses).
__device__ __forceinline__ void weno5b_masses_f32(const float* ar1, const float* ar2, const float* al1, int side,
                                                  float& a1r1_f, float& a2r2_f, float& alpha1_f) {
    float rL[2], rR[2], aL[2], aR[2], ac[2];
    float sumL = 0.0f, sumR = 0.0f;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float* fr = (k == 0) ? ar1 : ar2;
        float fa[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) fa[s] = (k == 0) ? al1[s] : 1.0f - al1[s];
        ac[k] = fa[2];
        float e[3], w[3], ea[3];
        weno5_f32_parts(fr[0], fr[1], fr[2], fr[3], fr[4], 1, e, w);
        weno5_f32_parts(fa[0], fa[1], fa[2], fa[3], fa[4], 1, ea, nullptr);
        rL[k] = fr[2] + __fmaf_rn(w[0], e[0], __fmaf_rn(w[1], e[1], w[2] * e[2]));
        aL[k] = fa[2] + __fmaf_rn(w[0], ea[0], __fmaf_rn(w[1], ea[1], w[2] * ea[2]));
        weno5_f32_parts(fr[0], fr[1], fr[2], fr[3], fr[4], -1, e, w);
        weno5_f32_parts(fa[0], fa[1], fa[2], fa[3], fa[4], -1, ea, nullptr);
        rR[k] = fr[2] + __fmaf_rn(w[0], e[0], __fmaf_rn(w[1], e[1], w[2] * e[2]));
        aR[k] = fa[2] + __fmaf_rn(w[0], ea[0], __fmaf_rn(w[1], ea[1], w[2] * ea[2]));
        const float th = fminf(bound_min_theta_f32(fr[2], rL[k], rR[k]), bound_min_theta_f32(fa[2], aL[k], aR[k]));
        rL[k] = __fmaf_rn(th, rL[k] - fr[2], fr[2]);
        aL[k] = __fmaf_rn(th, aL[k] - fa[2], fa[2]);
        rR[k] = __fmaf_rn(th, rR[k] - fr[2], fr[2]);
        aR[k] = __fmaf_rn(th, aR[k] - fa[2], fa[2]);
        sumL += aL[k];
        sumR += aR[k];
    }
    const float iL = 1.0f / sumL, iR = 1.0f / sumR;
    float Th = 1.0f;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float rc = (k == 0) ? ar1[2] : ar2[2];
        rL[k] *= iL;
        aL[k] *= iL;
        rR[k] *= iR;
        aR[k] *= iR;
        Th = fminf(Th, fminf(bound_min_theta_f32(rc, rL[k], rR[k]), bound_min_theta_f32(ac[k], aL[k], aR[k])));
    }
    const float r1 = (side == 1) ? rL[0] : rR[0];
    const float r2 = (side == 1) ? rL[1] : rR[1];
    const float a1 = (side == 1) ? aL[0] : aR[0];
    a1r1_f = __fmaf_rn(Th, r1 - ar1[2], ar1[2]);
    a2r2_f = __fmaf_rn(Th, r2 - ar2[2], ar2[2]);
    alpha1_f = __fmaf_rn(Th, a1 - al1[2], al1[2]);
}

// Bounded WENO face values of NP phases. WENO5B, ORDER 5:
// include/Operators_Compressible5Eq_NPhase/FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq_NPhase.H;
// WENO3B, ORDER 3: include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_WENO3B_D_Compressible5Eq.H:95-236,
// the six-equation and N-phase counterparts (same steps). Per phase: the WENO faces of alpha_k rho_k and of
// alpha_k (with the weights of alpha_k rho_k), one positivity theta for both; the faces divided by sum alpha_k;
// one common theta over all phases applied to the face of side `side`. r(k, s) and a(k, s) give alpha_k rho_k
// and alpha_k of stencil cell s = 0..ORDER-1 (centre ORDER/2); the results go to rf[k], af[k]. PT = double:
// the reference's arithmetic (quadrature weight 1/12 for ORDER 5, 1/6 for ORDER 3); PT = float: the mixed form.
// Wq > 0 replaces the quadrature weight (the bound-preserving path runs the fifth-order stencil with
// weight 1/6 for WENO3 / WENO3B, FiniteVolume_Parameter.H:114-127).
template <int NP, int ORDER, class PT, class FR, class FA>
__device__ __forceinline__ void bounded_phases(FR r, FA a, int side, PT* rf, PT* af, double Wq = 0.0) {
    constexpr bool F32 = std::is_same<PT, float>::value;
    constexpr int C = ORDER / 2;
    const double W = (Wq > 0.0) ? Wq : ((ORDER == 5) ? 1.0 / 12.0 : 1.0 / 6.0);
    PT rL[NP], rR[NP], aL[NP], aR[NP];
    PT sumL = 0, sumR = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        PT fr[ORDER], fa[ORDER];
#pragma unroll
        for (int s = 0; s < ORDER; ++s) {
            fr[s] = r(k, s);
            fa[s] = a(k, s);
        }
        PT th;
        if constexpr (F32 && ORDER == 3) {
            const float ra = fr[1] - fr[0], rb = fr[2] - fr[1], aa = fa[1] - fa[0], ab = fa[2] - fa[1];
            float w0 = weno3_w0_f32(ra, rb, 1);
            rL[k] = fr[1] + 0.5f * __fmaf_rn(w0, ra - rb, rb);
            aL[k] = fa[1] + 0.5f * __fmaf_rn(w0, aa - ab, ab);
            w0 = weno3_w0_f32(ra, rb, -1);
            rR[k] = fr[1] - 0.5f * __fmaf_rn(w0, ra - rb, rb);
            aR[k] = fa[1] - 0.5f * __fmaf_rn(w0, aa - ab, ab);
        } else if constexpr (!F32 && ORDER == 3) {
            double q[2], w[2], qa[2], wa[2];
            weno3_qw(fr[0], fr[1], fr[2], 1, q, w);
            rL[k] = weno3_sum(q, w);
            weno3_qw(fa[0], fa[1], fa[2], 1, qa, wa);
            aL[k] = weno3_sum(qa, w);
            weno3_qw(fr[0], fr[1], fr[2], -1, q, w);
            rR[k] = weno3_sum(q, w);
            weno3_qw(fa[0], fa[1], fa[2], -1, qa, wa);
            aR[k] = weno3_sum(qa, w);
        } else if constexpr (F32) {
            float e[3], w[3], ea[3];
            weno5_f32_parts(fr[0], fr[1], fr[2], fr[3], fr[4], 1, e, w);
            weno5_f32_parts(fa[0], fa[1], fa[2], fa[3], fa[4], 1, ea, nullptr);
            rL[k] = fr[2] + __fmaf_rn(w[0], e[0], __fmaf_rn(w[1], e[1], w[2] * e[2]));
            aL[k] = fa[2] + __fmaf_rn(w[0], ea[0], __fmaf_rn(w[1], ea[1], w[2] * ea[2]));
            weno5_f32_parts(fr[0], fr[1], fr[2], fr[3], fr[4], -1, e, w);
            weno5_f32_parts(fa[0], fa[1], fa[2], fa[3], fa[4], -1, ea, nullptr);
            rR[k] = fr[2] + __fmaf_rn(w[0], e[0], __fmaf_rn(w[1], e[1], w[2] * e[2]));
            aR[k] = fa[2] + __fmaf_rn(w[0], ea[0], __fmaf_rn(w[1], ea[1], w[2] * ea[2]));
        } else {
            double q[3], w[3], qa[3];
            weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], 1, q, w);
            rL[k] = weno_sum(q, w);
            weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], 1, qa, nullptr);
            aL[k] = weno_sum(qa, w);
            weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], -1, q, w);
            rR[k] = weno_sum(q, w);
            weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], -1, qa, nullptr);
            aR[k] = weno_sum(qa, w);
        }
        if constexpr (F32) {
            th = fminf(bound_min_theta_f32(fr[C], rL[k], rR[k], (float)W),
                       bound_min_theta_f32(fa[C], aL[k], aR[k], (float)W));
            rL[k] = __fmaf_rn(th, rL[k] - fr[C], fr[C]);
            aL[k] = __fmaf_rn(th, aL[k] - fa[C], fa[C]);
            rR[k] = __fmaf_rn(th, rR[k] - fr[C], fr[C]);
            aR[k] = __fmaf_rn(th, aR[k] - fa[C], fa[C]);
        } else {
            th = dmin(bound_min_theta(fr[C], rL[k], rR[k], W), bound_min_theta(fa[C], aL[k], aR[k], W));
            rL[k] = fr[C] + th * (rL[k] - fr[C]);
            aL[k] = fa[C] + th * (aL[k] - fa[C]);
            rR[k] = fr[C] + th * (rR[k] - fr[C]);
            aR[k] = fa[C] + th * (aR[k] - fa[C]);
        }
        sumL += aL[k];
        sumR += aR[k];
    }
    PT Th = 1;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const PT rc = r(k, C), ac = a(k, C);
        rL[k] /= sumL;
        aL[k] /= sumL;
        rR[k] /= sumR;
        aR[k] /= sumR;
        if constexpr (F32) {
            Th = fminf(Th, fminf(bound_min_theta_f32(rc, rL[k], rR[k], (float)W), bound_min_theta_f32(ac, aL[k], aR[k], (float)W)));
        } else {
            const double th_r = bound_min_theta(rc, rL[k], rR[k], W);
            const double th_a = bound_min_theta(ac, aL[k], aR[k], W);
            if (th_r < Th) Th = th_r;  // std::min({Th, th_r, th_a})
            if (th_a < Th) Th = th_a;
        }
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const PT rs = (side == 1) ? rL[k] : rR[k], as = (side == 1) ? aL[k] : aR[k];
        if constexpr (F32) {
            rf[k] = __fmaf_rn(Th, rs - r(k, C), r(k, C));
            af[k] = __fmaf_rn(Th, as - a(k, C), a(k, C));
        } else {
            rf[k] = r(k, C) + Th * (rs - r(k, C));
            af[k] = a(k, C) + Th * (as - a(k, C));
        }
    }
}

}  // namespace compas
