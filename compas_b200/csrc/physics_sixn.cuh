// Pointwise physics of the N-phase six-equation model in its internal-energy formulation
// (SIXEQS_IE_NPHASE) on the device.
//
// State U = (alpha_k, alpha_k rho_k, alpha_k rho_k e_k for k < NP, rho u_d, rho E), N = 3 NP + D + 1;
// primitives W = (alpha_k, alpha_k rho_k, alpha_k p_k, u_d, p) with p = sum_k alpha_k p_k. The phase
// pressures come from the phase internal energies (the total energy does not enter the primitives);
// the pressure relaxation after every stage resets the phase energies at the pressure of rho E. Sums
// over the phases start from 0.0 as the reference's loops do and every formula keeps the reference's
// association, so that the FP64 path reproduces the reference to the bit (no FMA contraction).
//
// Reference correspondence (file:line in the reference tree):
//   state layout        include/Physics_Compressible6Eq_IE_NPhase/Variables_Compressible6Eq_IE_NPhase.H
//   C2P / P2C / EOS     Conservative2Primitive_Compressible6Eq_IE_NPhase.H, Primitive2Conservative_...,
//                       EquationOfState_Phase_Compressible6Eq_IE_NPhase.H (NASG xi, phi = xi alpha)
//   sound speed         SoundSpeed_Compressible6Eq_IE_NPhase.H, rho_c2_Phase_..., rho_c2_Mixture_... (frozen)
//   physical flux       Conservative2Flux_Compressible6Eq_IE_NPhase.H
//   HLLC / LLF          Riemann_HLLC_Compressible6Eq_IE_NPhase.H, Riemann_LLF_Compressible6Eq_IE_NPhase.H
//                       (HLL is the generic form of riemann_llf_hll)
//   consistent limiter  include/Operators_Compressible6Eq_IE_NPhase/FVM_Reconstruction2Face_Conservative_LimiterConsistent_Compressible6Eq_IE_NPhase.H,
//                       FVM_Reconstruction2Face_LimiterConsistent_Compressible6Eq_IE_NPhase.H
//   relaxation          include/Physics_Compressible6Eq_IE_NPhase/RelaxationPressure_Instantaneous_Compressible6Eq_IE_NPhase.H
//                       (Newton iteration, admissibility, the safeguarded solve of
//                       include/RelaxationPressure_Safeguarded.H, phase energies at the pressure of rho E)
#pragma once

#include "physics.cuh"
#include "physics_nphase.cuh"
#include "relax.cuh"

namespace compas {

template <int DIM, int NPH>
struct SixEqN {
    static_assert(NPH >= 2 && NPH <= kMaxPhases, "2 <= NPHASE <= kMaxPhases");
    static constexpr int KIND = kModelSixN;
    static constexpr int D = DIM;
    static constexpr int NP = NPH;
    static constexpr int N = 3 * NPH + DIM + 1;
    static constexpr int NC = 1;            // FluxNC[0] = u*_n
    static constexpr int NCPF = 1;          // (no Phase-Field step in this engine)
    static constexpr int IA = 0;            // alpha_k at IA + k
    static constexpr int IR = NPH;          // alpha_k rho_k at IR + k
    static constexpr int IP = 2 * NPH;      // alpha_k rho_k e_k (state) / alpha_k p_k (primitive) at IP + k
    static constexpr int IM = 3 * NPH;      // rho u_d / u_d
    static constexpr int IE = 3 * NPH + DIM;  // rho E / p

    __device__ static __forceinline__ void cons2prim(double* W, const double* U, const Eos& e, unsigned int* err) {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += U[IR + k];
        double P = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double al = U[IA + k], ar = U[IR + k];
            const double xi = nasg_xi(al, ar, e.Ck[k], err);
            const double phi = xi * al;
            const double BP = phi * e.Bk[k];
            const double ard = ar * e.Dk[k];
            const double aps = ((U[IP + k] - ard) - BP) / (e.Ak[k] * xi);
            W[IA + k] = al;
            W[IR + k] = ar;
            W[IP + k] = aps;
            P += aps;
        }
#pragma unroll
        for (int d = 0; d < D; ++d) W[IM + d] = U[IM + d] / rho;
        W[IE] = P;
    }

    // Mixed precision: the phase pressures alpha_k p_k from the phase internal energies in FP64 (where the
    // energy cancels against the B_k term), the velocity by a near-FP64 reciprocal of rho (rcp_mixed), the
    // primitives rounded once to FP32. The FP32 WENO face states are converted back by prim2cons in FP64.
    __device__ static __forceinline__ void cons2prim_f32(float* W, const double* U, const Eos& e) {
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += U[IR + k];
        const double ir = rcp_mixed(rho);
        double P = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double al = U[IA + k], ar = U[IR + k];
            const double xi = nasg_xi(al, ar, e.Ck[k], nullptr);
            const double aps = ((U[IP + k] - ar * e.Dk[k]) - (xi * al) * e.Bk[k]) / (e.Ak[k] * xi);
            W[IA + k] = (float)al;
            W[IR + k] = (float)ar;
            W[IP + k] = (float)aps;
            P += aps;
        }
#pragma unroll
        for (int d = 0; d < D; ++d) W[IM + d] = (float)(U[IM + d] * ir);
        W[IE] = (float)P;
    }

    __device__ static __forceinline__ void prim2cons(double* U, const double* W, const Eos& e, unsigned int* err) {
        double rho = 0.0, rho_e = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double al = W[IA + k], ar = W[IR + k];
            rho += ar;
            const double xi = nasg_xi(al, ar, e.Ck[k], err);
            const double phi = xi * al;
            const double are = ((e.Ak[k] * xi) * W[IP + k] + phi * e.Bk[k]) + ar * e.Dk[k];
            U[IA + k] = al;
            U[IR + k] = ar;
            U[IP + k] = are;
            rho_e += are;
        }
#pragma unroll
        for (int d = 0; d < D; ++d) U[IM + d] = rho * W[IM + d];
        U[IE] = rho_e + (0.5 * rho) * ksum<D>(W + IM);
    }

    // Frozen mixture sound speed: rho c^2 = sum_k ((A_k + 1) alpha_k p_k + alpha_k B_k)/(A_k xi_k).
    __device__ static __forceinline__ double sound_speed(const double* W, const Eos& e, unsigned int* err) {
        double rc2 = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double xi = nasg_xi(W[IA + k], W[IR + k], e.Ck[k], err);
            rc2 += ((e.Ak[k] + 1.0) * W[IP + k] + W[IA + k] * e.Bk[k]) / (e.Ak[k] * xi);
        }
        double rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += W[IR + k];
        return sqrt(rc2 / rho);
    }

    // Physical flux in direction d: U V, plus p on the momentum and p V on the total energy.
    __device__ static __forceinline__ void flux(double* F, const double* U, const double* W, int d) {
        const double V = pick<D>(W + IM, d);
        const double p = W[IE];
#pragma unroll
        for (int i = 0; i < N; ++i) F[i] = U[i] * V;
#pragma unroll
        for (int c = 0; c < D; ++c)
            if (c == d) F[IM + c] = F[IM + c] + p;
        F[IE] = F[IE] + p * V;
    }

    __device__ static __forceinline__ double cmax_of(const double* WL, double cL, const double* WR, double cR) {
        return dmax(cL + sqrt(ksum<D>(WL + IM)), cR + sqrt(ksum<D>(WR + IM)));
    }

    // Local Lax-Friedrichs flux of the model: the wave-speed bound is the face's cmax.
    __device__ static __forceinline__ void llf(double* Fout, double* fnc, double& cmax, const double* UL,
                                               const double* UR, const Eos& e, int d, unsigned int* err) {
        double WL[N], WR[N], FL[N], FR[N];
        cons2prim(WL, UL, e, err);
        cons2prim(WR, UR, e, err);
        flux(FL, UL, WL, d);
        flux(FR, UR, WR, d);
        const double cL = sound_speed(WL, e, err);
        const double cR = sound_speed(WR, e, err);
        fnc[0] = 0.5 * (pick<D>(WL + IM, d) + pick<D>(WR + IM, d));
        cmax = cmax_of(WL, cL, WR, cR);
#pragma unroll
        for (int i = 0; i < N; ++i) Fout[i] = 0.5 * (FL[i] + FR[i]) - (0.5 * cmax) * (UR[i] - UL[i]);
    }

    // HLLC with the star states of the phase energies from the phase pressures
    // (Riemann_HLLC_Compressible6Eq_IE_NPhase.H: Q = F - S U, S* and p* from the mixture parts of Q).
    __device__ static __forceinline__ void hllc(double* Fout, double* fnc, double& cmax, const double* UL,
                                                const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
        (void)id_k;
        double WL[N], WR[N], FL[N], FR[N];
        cons2prim(WL, UL, e, err);
        cons2prim(WR, UR, e, err);
        flux(FL, UL, WL, d);
        flux(FR, UR, WR, d);
        const double cL = sound_speed(WL, e, err);
        const double cR = sound_speed(WR, e, err);
        const double VL = pick<D>(WL + IM, d), VR = pick<D>(WR + IM, d);
        const double V_avg = 0.5 * (VL + VR);
        const double c_avg = 0.5 * (cL + cR);
        const double SL = dmin(V_avg - c_avg, VL - cL);
        const double SR = dmax(V_avg + c_avg, VR + cR);
        const double Sm = dmin(0.0, SL);
        const double Sp = dmax(0.0, SR);
        double QL[N], QR[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            QR[i] = FR[i] - SR * UR[i];
            QL[i] = FL[i] - SL * UL[i];
        }
        double QL_rho = 0.0, QR_rho = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            QL_rho += QL[IR + k];
            QR_rho += QR[IR + k];
        }
        const double QLm = pick<D>(QL + IM, d), QRm = pick<D>(QR + IM, d);
        const double S_Star = (QLm - QRm) / (QL_rho - QR_rho);
        const double P_Star = -(QLm * QR_rho - QRm * QL_rho) / (QL_rho - QR_rho);
        const double sgn = sgn0(S_Star);
        // face velocity: the normal component from the star state, the tangential ones unchanged
        {
            const double fL = (SL - VL) / (SL - S_Star) - 1.0;
            const double fR = (SR - VR) / (SR - S_Star) - 1.0;
            fnc[0] = 0.5 * (1.0 + sgn) * (VL + Sm * fL) + 0.5 * (1.0 - sgn) * (VR + Sp * fR);
        }
        const double XiL = (VL - SL) / (S_Star - SL);
        const double XiR = (VR - SR) / (S_Star - SR);
        double UsL[N], UsR[N];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            UsL[IA + k] = QL[IA + k] / (S_Star - SL);
            UsR[IA + k] = QR[IA + k] / (S_Star - SR);
            UsL[IR + k] = QL[IR + k] / (S_Star - SL);
            UsR[IR + k] = QR[IR + k] / (S_Star - SR);
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double A = e.Ak[k], B = e.Bk[k], C = e.Ck[k];
            const double xiL = nasg_xi(WL[IA + k], WL[IR + k], C, err);
            const double xiR = nasg_xi(WR[IA + k], WR[IR + k], C, err);
            const double AxiL = A * xiL, AxiR = A * xiR;
            const double PhiL = xiL * WL[IA + k], PhiR = xiR * WR[IA + k];
            const double PhiLs = nasg_xi(UsL[IA + k], UsL[IR + k], C, err) * UsL[IA + k];
            const double PhiRs = nasg_xi(UsR[IA + k], UsR[IR + k], C, err) * UsR[IA + k];
            const double iXL = 1. / XiL, iXR = 1. / XiR;
            const double apL = (((AxiL * WL[IP + k] + PhiL * B) - (PhiLs * B) * iXL) - (0.5 * WL[IP + k]) * (iXL - 1.)) /
                               (AxiL + 0.5 * (iXL - 1.));
            const double apR = (((AxiR * WR[IP + k] + PhiR * B) - (PhiRs * B) * iXR) - (0.5 * WR[IP + k]) * (iXR - 1.)) /
                               (AxiR + 0.5 * (iXR - 1.));
            // EquationOfState_Phase (pressure to internal energy) of the star states
            const double xsL = nasg_xi(UsL[IA + k], UsL[IR + k], C, err);
            const double xsR = nasg_xi(UsR[IA + k], UsR[IR + k], C, err);
            UsL[IP + k] = ((A * xsL) * apL + (xsL * UsL[IA + k]) * B) + UsL[IR + k] * e.Dk[k];
            UsR[IP + k] = ((A * xsR) * apR + (xsR * UsR[IA + k]) * B) + UsR[IR + k] * e.Dk[k];
        }
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double vL = (c == d) ? S_Star : WL[IM + c];
            const double vR = (c == d) ? S_Star : WR[IM + c];
            UsL[IM + c] = vL * QL_rho / (S_Star - SL);
            UsR[IM + c] = vR * QR_rho / (S_Star - SR);
        }
        UsL[IE] = (QL[IE] - P_Star * S_Star) / (S_Star - SL);
        UsR[IE] = (QR[IE] - P_Star * S_Star) / (S_Star - SR);
#pragma unroll
        for (int i = 0; i < N; ++i)
            Fout[i] = 0.5 * (1.0 + sgn) * (FL[i] + Sm * (UsL[i] - UL[i])) + 0.5 * (1.0 - sgn) * (FR[i] + Sp * (UsR[i] - UR[i]));
        cmax = cmax_of(WL, cL, WR, cR);
    }

    // The consistent limiter of the MUSCL face state: the face state Uf back to primitives, the volume
    // fractions, partial densities and phase pressures re-reconstructed linearly from the cell's
    // primitives Wc (stride wstr) with one consistent factor per phase from the volume-fraction slopes;
    // velocity and mixture pressure keep the face values.
    template <class PT>
    __device__ static __forceinline__ void consistent_limit(double* Uf, const PT* Wc, int wstr, double dx, int side,
                                                            const Eos& e, unsigned int* err) {
        double Wf[N];
        cons2prim(Wf, Uf, e, err);
        const double den = ((double)side * 0.5) * dx;
        double s_ap[NP], s_ar[NP], s_al[NP], theta[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            s_ap[k] = (Wf[IP + k] - (double)Wc[(IP + k) * wstr]) / den;
            s_ar[k] = (Wf[IR + k] - (double)Wc[(IR + k) * wstr]) / den;
            s_al[k] = (Wf[IA + k] - (double)Wc[(IA + k) * wstr]) / den;
        }
        FiveEqN<DIM, NPH>::limiter_consistent(theta, s_al);
        const double sd = (double)side * 0.5;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            Wf[IP + k] = (double)Wc[(IP + k) * wstr] + (sd * (theta[k] * s_ap[k])) * dx;
            Wf[IR + k] = (double)Wc[(IR + k) * wstr] + (sd * (theta[k] * s_ar[k])) * dx;
            Wf[IA + k] = (double)Wc[(IA + k) * wstr] + (sd * (theta[k] * s_al[k])) * dx;
        }
        prim2cons(Uf, Wf, e, err);
    }

    // ---- instantaneous pressure relaxation of one cell (PressureRelaxation_Cell) --------------------
    __device__ static __forceinline__ double relax_f(double Pe, const double* Phi, const double* Pi, const Eos& e) {
        double fx = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double a = 1. + 1. / e.Ak[k];
            const double b = e.Bk[k] / e.Ak[k];
            fx += (Pi[k] - Phi[k] * Pe) / ((a * Pe + b) + 1.e-300);
        }
        return fx;
    }
    __device__ static __forceinline__ double relax_df(double Pe, const double* Phi, const double* Pi, const Eos& e) {
        double df = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double a = 1. + 1. / e.Ak[k];
            const double b = e.Bk[k] / e.Ak[k];
            const double t = (a * Pe + b) + 1.e-300;
            df += (-Phi[k] * b - Pi[k] * a) / (t * t);
        }
        return df;
    }
    // Newton iteration from |sum Pi| halved until f >= 0 (at most 10001 halvings), at most 51 updates.
    __device__ static __forceinline__ double relax_newton(const double* Phi, const double* Pi, const Eos& e) {
        double P0 = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) P0 += Pi[k];
        P0 = fabs(P0);
        double f0 = relax_f(P0, Phi, Pi, e);
        int nit = 0;
        while (f0 < 0 && P0 > 0) {
            P0 = 0.5 * P0;
            f0 = relax_f(P0, Phi, Pi, e);
            nit++;
            if (nit > 10000) break;
        }
        double Pe = P0;
        double fx = relax_f(Pe, Phi, Pi, e);
        int niter = 0;
        while (fabs(fx) > 1.e-16) {
            const double dfdx = relax_df(Pe, Phi, Pi, e);
            fx = relax_f(Pe, Phi, Pi, e);
            if (fabs(dfdx) < 1.e-14) break;
            Pe = Pe - fx / dfdx;
            niter++;
            if (niter > 50) break;
        }
        return Pe;
    }

    __device__ static __forceinline__ void relax(double* U, const Eos& e, double trace, unsigned int* err) {
        double W[N];
        cons2prim(W, U, e, err);
        bool nasg = false;
#pragma unroll
        for (int k = 0; k < NP; ++k) nasg = nasg || (e.Ck[k] > 0.0) || (e.Dk[k] != 0.0);
        double rho = 0.;
#pragma unroll
        for (int k = 0; k < NP; ++k) rho += W[IR + k];
        double Phi[NP], Pi[NP], Al[NP], Ar[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            Al[k] = W[IA + k];
            Ar[k] = W[IR + k];
            if (nasg) {
                Phi[k] = Al[k] - e.Ck[k] * Ar[k];
                Pi[k] = ((U[IP + k] - Ar[k] * e.Dk[k]) - Phi[k] * e.Bk[k]) / e.Ak[k];
            } else {
                Phi[k] = Al[k];
                Pi[k] = W[IP + k];
            }
        }
        const double Pe = relax_newton(Phi, Pi, e);
        double AlphaR[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double gamma = 1. + 1. / e.Ak[k];
            const double pinf = (gamma - 1.) * e.Bk[k] / gamma;
            if (nasg)
                AlphaR[k] = Al[k] + (Pi[k] - Phi[k] * Pe) / (gamma * (pinf + Pe));
            else
                AlphaR[k] = ((W[IP + k] + (Al[k] * gamma) * pinf) + (Al[k] * Pe) * (gamma - 1.)) / (gamma * (pinf + Pe));
        }
        const double fR = relax_f(Pe, Phi, Pi, e);
        bool admissible = finite_d(Pe) && (fabs(fR) <= 1.e-12);
        double Sum = 0.0, SumR = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            Sum += Al[k];
            SumR += AlphaR[k];
        }
        admissible = admissible && (fabs(SumR - Sum) <= 1.e-12);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            admissible = admissible && finite_d(AlphaR[k]);
            if (Al[k] > 0.0) {
                const double pinf_k = e.Bk[k] / (e.Ak[k] + 1.0);
                admissible = admissible && (Pe + pinf_k > 0.0) && (Al[k] > trace);
            }
        }
        if (!admissible) {
            const int path = relax_safeguarded<NP>(AlphaR, Al, Ar, Phi, Pi, e.Ak, e.Bk, trace);
            if (path == kPathNoRoot) flag_error(err, COMPAS_B200_ERR_RELAX_NOROOT);
        }
        const double rhoe_h = U[IE] - (0.5 * rho) * ksum<D>(W + IM);
        double AreR[NP];
        if (nasg) {
            double sum_BPhi = 0.0, sum_APhi = 0.0, sum_q = 0.0, PhiR[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                PhiR[k] = nasg_xi(AlphaR[k], Ar[k], e.Ck[k], err) * AlphaR[k];
                sum_BPhi += PhiR[k] * e.Bk[k];
                sum_APhi += PhiR[k] * e.Ak[k];
                sum_q += Ar[k] * e.Dk[k];
            }
            const double pr = ((rhoe_h - sum_q) - sum_BPhi) / sum_APhi;
#pragma unroll
            for (int k = 0; k < NP; ++k) AreR[k] = PhiR[k] * (e.Ak[k] * pr + e.Bk[k]) + Ar[k] * e.Dk[k];
        } else {
            double a = 0., b = 0., dsum = 0.;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                a += AlphaR[k] * e.Bk[k];
                b += AlphaR[k] * e.Ak[k];
                if (e.Dk[k] != 0.0) dsum += Ar[k] * e.Dk[k];
            }
            const double pr = ((rhoe_h - a) - dsum) / b;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                AreR[k] = AlphaR[k] * (e.Ak[k] * pr + e.Bk[k]);
                if (e.Dk[k] != 0.0) AreR[k] += Ar[k] * e.Dk[k];
            }
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            U[IA + k] = AlphaR[k];
            U[IP + k] = AreR[k];
        }
    }
};

}  // namespace compas
