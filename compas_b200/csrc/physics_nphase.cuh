// Pointwise physics of the N-phase five-equation model (FIVEEQS_NPHASE) on the device.
//
// State U = (alpha_k rho_k for k < NP, rho u_d, rho E, alpha_k for k < NP), N = 2 NP + D + 1;
// primitives W = (alpha_k rho_k, u_d, p, alpha_k). The mixture EOS sums over the phases start from
// 0.0 as the reference's loops do, and every formula keeps the reference's association, so that the
// plain FP64 path reproduces the reference to the bit (the library is compiled without FMA
// contraction).
//
// Reference correspondence (file:line in the reference tree):
//   state layout        include/Physics_Compressible5Eq_NPhase/Variables_Compressible5Eq_NPhase.H
//   C2P / P2C / EOS     include/Physics_Compressible5Eq_NPhase/Conservative2Primitive_Compressible5Eq_NPhase.H,
//                       Primitive2Conservative_Compressible5Eq_NPhase.H, EquationOfState_Mixture_Compressible5Eq_NPhase.H
//   sound speed         SoundSpeed_Compressible5Eq_NPhase.H, rho_c2_Mixture_Compressible5Eq_NPhase.H,
//                       rho_c2_Phase_Compressible5Eq_NPhase.H
//   physical flux       Conservative2Flux_Compressible5Eq_NPhase.H
//   HLLC                Riemann_HLLC_Compressible5Eq_NPhase.H
//   Kapila factors      NonConservative_Compressible5Eq_NPhase.H, Conservative2K_Compressible5Eq_NPhase.H,
//                       include/Operators_Compressible5Eq_NPhase/FVM_SurfaceIntegralNC_Compressible5Eq_NPhase.H
//   consistent limiter  include/Operators_Compressible5Eq_NPhase/FVM_Reconstruction2Face_Conservative_LimiterConsistent_Compressible5Eq_NPhase.H,
//                       FVM_Reconstruction2Face_LimiterConsistent_Compressible5Eq_NPhase.H,
//                       include/Operators_FV/Limiter_Consistent.H, Reconstruction2Face_Linear.H
#pragma once

#include "physics.cuh"

namespace compas {

template <int DIM, int NPH>
struct FiveEqN {
    static_assert(NPH >= 2 && NPH <= kMaxPhases, "2 <= NPHASE <= kMaxPhases");
    static constexpr int KIND = kModelFiveN;
    static constexpr int D = DIM;
    static constexpr int NP = NPH;
    static constexpr int N = 2 * NPH + DIM + 1;
    static constexpr int NC = 1;             // FluxNC[0] = u*_n
    static constexpr int NCPF = 1;           // (no Phase-Field step in this engine)
    static constexpr int IR = 0;             // alpha_k rho_k at IR + k
    static constexpr int IM = NPH;           // rho u_d (u_d among the primitives)
    static constexpr int IE = NPH + DIM;     // rho E (p among the primitives)
    static constexpr int IA = NPH + DIM + 1; // alpha_1; alpha_k at IA + k

    // EquationOfState_Mixture sums: rho D, A_P = sum phi_k A_k, B_P = sum phi_k B_k.
    __device__ static __forceinline__ void mix_sums(const double* ar, const double* al, const Eos& e, double& rho_D,
                                                    double& AP, double& BP, unsigned int* err) {
        rho_D = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho_D += ar[k] * e.Dk[k];
        AP = 0.0;
        BP = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double phi = nasg_phi(al[k], ar[k], e.Ck[k], err);
            AP += phi * e.Ak[k];
            BP += phi * e.Bk[k];
        }
    }

    __device__ static __forceinline__ void cons2prim(double* W, const double* U, const Eos& e, unsigned int* err) {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += U[k];
        double u[3];
#pragma unroll
        for (int d = 0; d < D; ++d) u[d] = U[IM + d] / rho;
        const double rho_e = U[IE] - (0.5 * rho) * ksum<D>(u);
        double rho_D, AP, BP;
        mix_sums(U, U + IA, e, rho_D, AP, BP, err);
#pragma unroll
        for (int k = 0; k < NP; ++k) W[k] = U[k];
#pragma unroll
        for (int d = 0; d < D; ++d) W[IM + d] = u[d];
        W[IE] = ((rho_e - rho_D) - BP) / AP;
#pragma unroll
        for (int k = 0; k < NP; ++k) W[IA + k] = U[IA + k];
    }

    // Mixed precision: the pressure numerator rho e - rho D - B_P (where the energy cancels against
    // the B_k terms) and A_P in FP64, near-FP64 reciprocals (rcp_mixed), the primitives rounded once to FP32.
    __device__ static __forceinline__ void cons2prim_f32(float* W, const double* U, const Eos& e) {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += U[k];
        const double ir = rcp_mixed(rho);
        double m2 = U[IM] * U[IM] + U[IM + 1] * U[IM + 1];
        if (D == 3) m2 += U[IM + 2] * U[IM + 2];
        double rho_D = 0.0, AP = 0.0, BP = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double al = U[IA + k];
            const double phi = (e.Ck[k] > 0.0) ? al - e.Ck[k] * U[k] : al;
            rho_D += U[k] * e.Dk[k];
            AP += phi * e.Ak[k];
            BP += phi * e.Bk[k];
        }
        const double num = ((U[IE] - 0.5 * m2 * ir) - rho_D) - BP;
#pragma unroll
        for (int k = 0; k < NP; ++k) W[k] = (float)U[k];
#pragma unroll
        for (int d = 0; d < D; ++d) W[IM + d] = (float)(U[IM + d] * ir);
        W[IE] = (float)(num * rcp_mixed(AP));
#pragma unroll
        for (int k = 0; k < NP; ++k) W[IA + k] = (float)U[IA + k];
    }

    __device__ static __forceinline__ void prim2cons(double* U, const double* W, const Eos& e, unsigned int* err) {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += W[k];
        double rho_D, AP, BP;
        mix_sums(W, W + IA, e, rho_D, AP, BP, err);
        const double rho_e = (AP * W[IE] + BP) + rho_D;
#pragma unroll
        for (int k = 0; k < NP; ++k) U[k] = W[k];
#pragma unroll
        for (int d = 0; d < D; ++d) U[IM + d] = rho * W[IM + d];
        U[IE] = rho_e + (0.5 * rho) * ksum<D>(W + IM);
#pragma unroll
        for (int k = 0; k < NP; ++k) U[IA + k] = W[IA + k];
    }

    // rho_c2_Phase: gamma_k (p + pinf_k) = ((A_k + 1) p + B_k)/A_k.
    __device__ static __forceinline__ double rc2_phase(double p, const Eos& e, int k) {
        return ((e.Ak[k] + 1.0) * p + e.Bk[k]) / e.Ak[k];
    }

    // rho_c2_Mixture: K = 0 sum (alpha_k A_k) rc2_k / A_P; K = 1 Wood, 1 / sum phi_k / rc2_k.
    __device__ static __forceinline__ double rho_c2_mix(const double* W, const double* rc2, const Eos& e, int id_k,
                                                        unsigned int* err) {
        if (id_k == 0) {
            double num = 0.0, AP = 0.0;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const double phi = nasg_phi(W[IA + k], W[k], e.Ck[k], err);
                num += (W[IA + k] * e.Ak[k]) * rc2[k];
                AP += phi * e.Ak[k];
            }
            return num / AP;
        }
        double inv = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) inv += nasg_phi(W[IA + k], W[k], e.Ck[k], err) / rc2[k];
        return 1.0 / inv;
    }

    __device__ static __forceinline__ double sound_speed(const double* W, const Eos& e, int id_k, unsigned int* err) {
        double rc2[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) rc2[k] = rc2_phase(W[IE], e, k);
        const double rho_c2 = rho_c2_mix(W, rc2, e, id_k, err);
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += W[k];
        return sqrt(rho_c2 / rho);
    }

    // Kapila factors phi_k (1 + K_k) of the alpha_k equations from the cell primitives
    // (FVM_SurfaceIntegral_NC: alpha_k += phi_k (1 + K_k) div u*; phi_k = alpha_k unless K = 1).
    __device__ static __forceinline__ void kapila_factors(double* fac, const double* W, const Eos& e, int id_k,
                                                          unsigned int* err) {
        if (id_k == 1) {
            double rc2[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) rc2[k] = rc2_phase(W[IE], e, k);
            const double rho_c2 = rho_c2_mix(W, rc2, e, 1, err);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const double K = rho_c2 / rc2[k] - 1.0;
                fac[k] = nasg_phi(W[IA + k], W[k], e.Ck[k], err) * (1.0 + K);
            }
        } else {
#pragma unroll
            for (int k = 0; k < NP; ++k) fac[k] = W[IA + k] * (1.0 + 0.0);
        }
    }

    __device__ static __forceinline__ void flux(double* F, const double* U, const double* W, int d) {
        const double V = pick<D>(W + IM, d);
        const double p = W[IE];
#pragma unroll
        for (int k = 0; k < NP; ++k) F[k] = U[k] * V;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            F[IM + c] = U[IM + c] * V;
            if (c == d) F[IM + c] = F[IM + c] + p;
        }
        F[IE] = (U[IE] + p) * V;
#pragma unroll
        for (int k = 0; k < NP; ++k) F[IA + k] = U[IA + k] * V;
    }

    __device__ static __forceinline__ void hllc(double* Fout, double* fnc, double& cmax, const double* UL,
                                                const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
        double WL[N], WR[N];
        cons2prim(WL, UL, e, err);
        cons2prim(WR, UR, e, err);
        double FL[N], FR[N];
        flux(FL, UL, WL, d);
        flux(FR, UR, WR, d);
        const double cL = sound_speed(WL, e, id_k, err);
        const double cR = sound_speed(WR, e, id_k, err);
        const double VL = pick<D>(WL + IM, d), VR = pick<D>(WR + IM, d);
        const double pL = WL[IE], pR = WR[IE];
        const double V_avg = 0.5 * (VL + VR);
        const double c_avg = 0.5 * (cL + cR);
        const double SL = dmin(V_avg - c_avg, VL - cL);
        const double SR = dmax(V_avg + c_avg, VR + cR);
        const double Sm = dmin(0.0, SL);
        const double Sp = dmax(0.0, SR);
        double rhoL = 0.0, rhoR = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            rhoL += WL[k];
            rhoR += WR[k];
        }
        const double S_Star = (((pR - pL) + (rhoL * VL) * (SL - VL)) - (rhoR * VR) * (SR - VR)) /
                              (rhoL * (SL - VL) - rhoR * (SR - VR));
        const double s = sgn0(S_Star);
        const double hp = 0.5 * (1.0 + s), hm = 0.5 * (1.0 - s);
        const double fL = (SL - VL) / (SL - S_Star);
        const double fR = (SR - VR) / (SR - S_Star);
        double vel = hp * VL + hm * VR;
        vel = vel + ((hp * Sm) * (fL - 1.0) + (hm * Sp) * (fR - 1.0));
        fnc[0] = vel;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double sL = fL * UL[i];
            double sR = fR * UR[i];
            if (i == IM + d) {
                sL = sL + (fL * rhoL) * (S_Star - VL);
                sR = sR + (fR * rhoR) * (S_Star - VR);
            } else if (i == IE) {
                sL = sL + (fL * (S_Star - VL)) * (rhoL * S_Star + pL / (SL - VL));
                sR = sR + (fR * (S_Star - VR)) * (rhoR * S_Star + pR / (SR - VR));
            }
            Fout[i] = hp * (FL[i] + Sm * (sL - UL[i])) + hm * (FR[i] + Sp * (sR - UR[i]));
        }
        const double qL = cL + sqrt(ksum<D>(WL + IM));
        const double qR = cR + sqrt(ksum<D>(WR + IM));
        cmax = dmax(qL, qR);
    }

    // Limiter_Consistent: one factor per phase from the volume-fraction slopes so that the limited
    // volume fractions keep summing to what the unlimited ones sum to. The largest |slope| is the
    // first maximum (std::max_element).
    __device__ static __forceinline__ void limiter_consistent(double* theta, const double* slope) {
        const double ep = 1.0e-10;
        double sum = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) sum += slope[k];
        int imax = 0;
        double amax = fabs(slope[0]);
#pragma unroll
        for (int k = 1; k < NP; ++k) {
            const double a = fabs(slope[k]);
            if (amax < a) {
                amax = a;
                imax = k;
            }
        }
        double smax = slope[0];
#pragma unroll
        for (int k = 1; k < NP; ++k)
            if (k == imax) smax = slope[k];
        if (fabs(smax) < ep || fabs(sum) < ep) {
#pragma unroll
            for (int k = 0; k < NP; ++k) theta[k] = 1.0;
        } else {
            const double smaxS = smax - sum;
            const double t_other = dmax(dmin(smax / smaxS, 1.0), 0.0);
            const double t_max = dmax(dmin(smaxS / smax, 1.0), 0.0);
#pragma unroll
            for (int k = 0; k < NP; ++k) theta[k] = (k == imax) ? t_max : t_other;
        }
    }

    // FVM_Reconstruction2Face_Conservative_LimiterConsistent: the face state Uf (from the WENO5
    // primitives) is converted back to primitives, the partial densities and volume fractions are
    // re-reconstructed linearly from the stencil centre c (primitives Wc: masses at 0.., volume
    // fractions at IA..) with the consistent factors of the volume-fraction slopes, and the face state
    // is rebuilt; velocity and pressure keep the face values. side = +1 for the left state of a face
    // (centre = the cell below it), -1 for the right state.
    template <class PT>
    __device__ static __forceinline__ void consistent_limit(double* Uf, const PT* Wc, int wstr, double dx, int side,
                                                            const Eos& e, unsigned int* err) {
        double Wf[N];
        cons2prim(Wf, Uf, e, err);
        const double sd = (double)side * 0.5;
        const double den = sd * dx;
        double s_ar[NP], s_al[NP], theta[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            s_ar[k] = (Wf[k] - (double)Wc[k * wstr]) / den;
            s_al[k] = (Wf[IA + k] - (double)Wc[(IA + k) * wstr]) / den;
        }
        limiter_consistent(theta, s_al);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            Wf[k] = (double)Wc[k * wstr] + (sd * (theta[k] * s_ar[k])) * dx;
            Wf[IA + k] = (double)Wc[(IA + k) * wstr] + (sd * (theta[k] * s_al[k])) * dx;
        }
        prim2cons(Uf, Wf, e, err);
    }
};

}  // namespace compas
