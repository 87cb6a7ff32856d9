// Phase-Field regularisation flux of one face from the reconstructed face states and the face gradient
// of the regularisation potential Q, with the upwind/downwind (PhaseField.ID_Flux = 0) or the HLL (1)
// phase fluxes, in the phasic (PhaseField.ID_FluxPhase2Flux = 0) or the mixture (1) formulation;
// SIXEQS with the non-conservative face terms of its phase-energy exchange.
//
// Reference (FIVEEQS):
//   FVM_Conservative2FluxPhaseField_K  include/Operators_Compressible5Eq_PhaseField/FVM_Conservative2FluxPhaseField_K_Compressible5Eq_PhaseField.H:15-69
//   FluxPhaseField                     include/Physics_Compressible5Eq_PhaseField/FluxPhaseField_Compressible5Eq_PhaseField.H
//   phase fluxes J_k rho_k, J_k (UD)   include/Physics_Compressible_TwoPhase_PhaseField/FluxPhasePhaseField_UD_Compressible_TwoPhase_PhaseField.H
//   mixture flux                       include/Physics_Compressible5Eq_PhaseField/FluxPhaseField_Mixture_Compressible5Eq_PhaseField.H
//   phasic face states                 include/Physics_Compressible5Eq/Conservative2ConservativePhase_Compressible5Eq.H
//                                      (phase energies from the pressure, clipped at the p_min energies)
//   phasic formulation                 include/Physics_Compressible5Eq/VectorPhase2Vector_Compressible5Eq.H
//   phase fluxes (HLL)                 include/Physics_Compressible_TwoPhase_PhaseField/FluxPhasePhaseField_HLL_Compressible_TwoPhase_PhaseField.H,
//                                      ConservativePhase2FluxPhasePhaseField_Compressible_TwoPhase_PhaseField.H
//   f_Upwind / f_Downwind              include/Operators_FV/f_Upwind.H, f_Downwind.H
// Reference (SIXEQS):
//   FVM_Conservative2FluxPhaseField_K  include/Operators_Compressible6Eq_PhaseField/FVM_Conservative2FluxPhaseField_K_Compressible6Eq_PhaseField.H:13-66
//   FluxPhaseField                     include/Physics_Compressible6Eq_PhaseField/FluxPhaseField_Compressible6Eq_PhaseField.H:10-72
//   phasic face states                 include/Physics_Compressible6Eq/Conservative2ConservativePhase_Compressible6Eq.H
//   phase fluxes (UD), FluxNC terms    include/Physics_Compressible6Eq_PhaseField/FluxPhasePhaseField_UD_Compressible6Eq_PhaseField.H
//   phase fluxes (HLL), FluxNC terms   include/Physics_Compressible6Eq_PhaseField/FluxPhasePhaseField_HLL_Compressible6Eq_PhaseField.H,
//                                      ConservativePhase2FluxPhasePhaseField_Compressible6Eq_PhaseField.H
//   phasic formulation                 include/Physics_Compressible6Eq/VectorPhase2Vector_Compressible6Eq.H
//   mixture formulation                include/Physics_Compressible6Eq_PhaseField/FluxPhaseField_Mixture_Compressible6Eq_PhaseField.H
// The flux is stored negated (the face array of PhaseField_ComputeFaceFluxes holds -fhat,
// source/Class_Compressible_PhaseField.cpp:770-855), so the stage kernel's surface integral applies.
#pragma once

namespace compas {

__device__ __forceinline__ double f_upwind(double fL, double fR, double V) {
    return (V > 0.0) ? fL : ((V < 0.0) ? fR : 0.5 * (fL + fR));
}
__device__ __forceinline__ double f_downwind(double fL, double fR, double V) {
    return (V > 0.0) ? fR : ((V < 0.0) ? fL : 0.5 * (fL + fR));
}

// HLL phase flux of the Phase-Field step: with the phase velocities V1 = alpha2 G, V2 = -alpha1 G of
// both sides, Sp = max(0, -V1L, -V2L, -V1R, -V2R) + 1e-10 and Sm = min(...) - 1e-10 (std::max / std::min
// over the list, first extremum kept), and F = (Sp FL - Sm FR - Sp Sm (CR - CL)) / (Sp - Sm) per phase
// quantity C with phase flux C V.
struct PfHll {
    double V1L, V2L, V1R, V2R, Sp, Sm, SpSm, den;
    __device__ __forceinline__ PfHll(double a1L, double a1R, double gq) {
        const double g1 = gq, g2 = -g1;
        V1L = (1.0 - a1L) * g1;
        V2L = a1L * g2;
        V1R = (1.0 - a1R) * g1;
        V2R = a1R * g2;
        const double c[4] = {-V1L, -V2L, -V1R, -V2R};
        double mx = 0.0, mn = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            mx = (mx < c[i]) ? c[i] : mx;
            mn = (c[i] < mn) ? c[i] : mn;
        }
        Sp = mx + 1.0e-10;
        Sm = mn - 1.0e-10;
        SpSm = Sp * Sm;
        den = Sp - Sm;
    }
    // phase 1 (velocity V1) and phase 2 (V2) quantity with states cl, cr
    __device__ __forceinline__ double p1(double cl, double cr) const {
        return (Sp * (cl * V1L) - Sm * (cr * V1R) - SpSm * (cr - cl)) / den;
    }
    __device__ __forceinline__ double p2(double cl, double cr) const {
        return (Sp * (cl * V2L) - Sm * (cr * V2R) - SpSm * (cr - cl)) / den;
    }
};

// Q gradient of the face of direction d at (i,j,k) (face arrays nodal in d, x fastest).
__device__ __forceinline__ double pf_face_gq(const StageArgs& a, int d, int i, int j, int k) {
    const int n0 = a.g.n[0], n1 = a.g.n[1];
    long long q;
    if (d == 0) q = (long long)i + (long long)(n0 + 1) * ((long long)j + (long long)n1 * k);
    else if (d == 1) q = (long long)i + (long long)n0 * ((long long)j + (long long)(n1 + 1) * k);
    else q = (long long)i + (long long)n0 * ((long long)j + (long long)n1 * k);
    return a.gq[d][q];
}

// MIX: the mixed form takes the face velocities and pressures from the FP32 primitives (the
// phase-field flux arithmetic is FP32-grade there; the masses and volume fractions stay the FP64 face
// states); the plain form converts in FP64 as the reference does.
template <int D, bool MIX = false>
__device__ __forceinline__ void pf_face_flux(double* F, const double* UL, const double* UR, double gq, const Eos& e,
                                             int phasic, int hll, unsigned int* err) {
    using M = FiveEq<D>;
    constexpr int N = M::N;
    // phase fluxes (the two phases carry Q and -Q) of the masses and volume fractions
    const double g1 = gq, g2 = -g1;
    const double a1L = UL[M::IA], a1R = UR[M::IA];
    const double a2L = 1.0 - a1L, a2R = 1.0 - a1R;
    double J1r1, J2r2, J1, J2;
    if (hll) {
        const PfHll h(a1L, a1R, gq);
        J1r1 = h.p1(UL[0], UR[0]);
        J2r2 = h.p2(UL[1], UR[1]);
        J1 = h.p1(a1L, a1R);
        J2 = h.p2(a2L, a2R);
    } else {
        const double a2u = f_upwind(a2L, a2R, g1);
        const double a1u = f_upwind(a1L, a1R, g2);
        J1r1 = f_downwind(UL[0], UR[0], g1) * a2u * g1;
        J2r2 = f_downwind(UL[1], UR[1], g2) * a1u * g2;
        J1 = f_downwind(a1L, a1R, g1) * a2u * g1;
        J2 = f_downwind(a2L, a2R, g2) * a1u * g2;
    }
    // mixture fluxes of momentum and energy
    double WL[N], WR[N];
    if constexpr (MIX) {
        float wl[N], wr[N];
        M::cons2prim_f32(wl, UL, e);
        M::cons2prim_f32(wr, UR, e);
#pragma unroll
        for (int n = 0; n < N; ++n) {
            WL[n] = wl[n];
            WR[n] = wr[n];
        }
    } else {
        M::cons2prim(WL, UL, e, err);
        M::cons2prim(WR, UR, e, err);
    }
    if (phasic) {
        // phasic states: alpha_k rho_k e_k from the face pressure, clipped at the energy of p_min_k with
        // the mixture internal energy kept; alpha_k rho_k u; alpha_k rho_k E_k
        double m1[2][3], m2[2][3], E1[2], E2[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double* U = s ? UR : UL;
            const double* W = s ? WR : WL;
            const double r1 = U[0], r2 = U[1], a1 = U[M::IA], a2 = 1.0 - a1, p = W[M::IE];
            const double phi1 = nasg_phi(a1, r1, e.C1, err), phi2 = nasg_phi(a2, r2, e.C2, err);
            double e1 = phi1 * e.A1 * p + phi1 * e.B1 + r1 * e.D1;
            const double e1m = phi1 * e.A1 * e.pmin1 + phi1 * e.B1 + r1 * e.D1;
            double e2 = phi2 * e.A2 * p + phi2 * e.B2 + r2 * e.D2;
            const double e2m = phi2 * e.A2 * e.pmin2 + phi2 * e.B2 + r2 * e.D2;
            const double re = e1 + e2;
            if (e1 < e1m) {
                e1 = e1m;
                e2 = re - e1;
            } else if (e2 < e2m) {
                e2 = e2m;
                e1 = re - e2;
            }
            const double k = ksum<D>(W + 2);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                m1[s][c] = r1 * W[2 + c];
                m2[s][c] = r2 * W[2 + c];
            }
            E1[s] = e1 + (0.5 * r1) * k;
            E2[s] = e2 + (0.5 * r2) * k;
        }
        const double a2u = f_upwind(a2L, a2R, g1);
        const double a1u = f_upwind(a1L, a1R, g2);
        const PfHll h(a1L, a1R, gq);
        auto j1 = [&](double l, double r) { return hll ? h.p1(l, r) : f_downwind(l, r, g1) * a2u * g1; };
        auto j2 = [&](double l, double r) { return hll ? h.p2(l, r) : f_downwind(l, r, g2) * a1u * g2; };
        F[0] = -J1r1;
        F[1] = -J2r2;
#pragma unroll
        for (int c = 0; c < D; ++c) F[2 + c] = -(j1(m1[0][c], m1[1][c]) + j2(m2[0][c], m2[1][c]));
        F[M::IE] = -(j1(E1[0], E1[1]) + j2(E2[0], E2[1]));
        F[M::IA] = -J1;
        return;
    }
    const double Mf = J1r1 + J2r2;
    double ud[3];
#pragma unroll
    for (int c = 0; c < D; ++c) ud[c] = f_downwind(WL[2 + c], WR[2 + c], Mf);
    const double eK = 0.5 * ksum<D>(ud);
    const double MeK = Mf * eK;
    const double p1 = f_downwind(WL[M::IE], WR[M::IE], J1);
    const double J1phi = (e.C1 > 0.0) ? J1 - e.C1 * J1r1 : J1;
    const double J1r1e1 = e.A1 * J1phi * p1 + e.B1 * J1phi + e.D1 * J1r1;
    const double p2 = f_downwind(WL[M::IE], WR[M::IE], J2);
    const double J2phi = (e.C2 > 0.0) ? J2 - e.C2 * J2r2 : J2;
    const double J2r2e2 = e.A2 * J2phi * p2 + e.B2 * J2phi + e.D2 * J2r2;
    F[0] = -J1r1;
    F[1] = -J2r2;
#pragma unroll
    for (int c = 0; c < D; ++c) F[2 + c] = -(Mf * ud[c]);
    F[M::IE] = -(MeK + J1r1e1 + J2r2e2);
    F[M::IA] = -J1;
}

// SIXEQS: F (stored negated) and the four non-conservative face terms fnc = (J1 rho1, J2 rho2,
// J1 rho1 EK, J2 rho2 EK). phasic: 1 the phasic formulation (each phase's mass, momentum, energy and
// volume fraction carried by its own flux), 0 the mixture formulation. MIX as in pf_face_flux: the face
// velocities and phase pressures come from the FP32 primitives, the masses and volume fraction stay the
// FP64 face states.
template <int D, bool MIX = false>
__device__ __forceinline__ void pf_face_flux_six(double* F, double* fnc, const double* UL, const double* UR, double gq,
                                                 const Eos& e, int phasic, int hll, unsigned int* err) {
    using M = SixEq<D>;
    constexpr int N = M::N;
    double W[2][N];
    if constexpr (MIX) {
        float w[N];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double* U = s ? UR : UL;
            M::cons2prim_f32(w, U, e);
#pragma unroll
            for (int n = 0; n < N; ++n) W[s][n] = w[n];
            W[s][0] = U[0];
            W[s][1] = U[1];
            W[s][M::IA] = U[M::IA];
        }
    } else {
        M::cons2prim(W[0], UL, e, err);
        M::cons2prim(W[1], UR, e, err);
    }
    // phasic states of the two sides: alpha_k rho_k, alpha_k rho_k u_d, alpha_k rho_k E_k, alpha_k
    double r1[2], r2[2], m1[2][3], m2[2][3], E1[2], E2[2], a1[2], a2[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        a1[s] = W[s][M::IA];
        a2[s] = 1.0 - a1[s];
        r1[s] = W[s][0];
        r2[s] = W[s][1];
        const double e1 = M::phase_e(W[s][M::IE1], a1[s], r1[s], e.A1, e.B1, e.C1, e.D1, err);
        const double e2 = M::phase_e(W[s][M::IE2], a2[s], r2[s], e.A2, e.B2, e.C2, e.D2, err);
        const double k = ksum<D>(W[s] + 2);
#pragma unroll
        for (int c = 0; c < D; ++c) {
            m1[s][c] = r1[s] * W[s][2 + c];
            m2[s][c] = r2[s] * W[s][2 + c];
        }
        E1[s] = e1 + (0.5 * r1[s]) * k;
        E2[s] = e2 + (0.5 * r2[s]) * k;
    }
    // phase fluxes: phase 1 carries Q, phase 2 -Q; UD: each weighted by the upwind volume fraction of
    // the other phase and the downwind value of the carried quantity; HLL: PfHll
    const double g1 = gq, g2 = -g1;
    const double a2u = f_upwind(a2[0], a2[1], g1);
    const double a1u = f_upwind(a1[0], a1[1], g2);
    const PfHll h(a1[0], a1[1], gq);
    auto j1 = [&](double l, double r) { return hll ? h.p1(l, r) : f_downwind(l, r, g1) * a2u * g1; };
    auto j2 = [&](double l, double r) { return hll ? h.p2(l, r) : f_downwind(l, r, g2) * a1u * g2; };
    const double J1r1 = j1(r1[0], r1[1]);
    const double J2r2 = j2(r2[0], r2[1]);
    // kinetic energy per unit mass of the mixture velocity of the phasic states
    double uL[3], uR[3];
#pragma unroll
    for (int c = 0; c < D; ++c) {
        uL[c] = (m1[0][c] + m2[0][c]) / (r1[0] + r2[0]);
        uR[c] = (m1[1][c] + m2[1][c]) / (r1[1] + r2[1]);
    }
    const double EKL = 0.5 * ksum<D>(uL), EKR = 0.5 * ksum<D>(uR);
    fnc[0] = J1r1;
    fnc[1] = J2r2;
    fnc[2] = j1(r1[0] * EKL, r1[1] * EKR);
    fnc[3] = j2(r2[0] * EKL, r2[1] * EKR);
    const double J1 = j1(a1[0], a1[1]);
    const double J2 = j2(a2[0], a2[1]);
    F[0] = -J1r1;
    F[1] = -J2r2;
    F[M::IA] = -J1;
    if (phasic) {
#pragma unroll
        for (int c = 0; c < D; ++c) F[2 + c] = -(j1(m1[0][c], m1[1][c]) + j2(m2[0][c], m2[1][c]));
        F[M::IE1] = -j1(E1[0], E1[1]);
        F[M::IE2] = -j2(E2[0], E2[1]);
    } else {
        const double Mf = J1r1 + J2r2;
        double ud[3];
#pragma unroll
        for (int c = 0; c < D; ++c) ud[c] = f_downwind(W[0][2 + c], W[1][2 + c], Mf);
        const double eK = 0.5 * ksum<D>(ud);
        const double pL = W[0][M::IE1] + W[0][M::IE2], pR = W[1][M::IE1] + W[1][M::IE2];
        const double p1 = f_downwind(pL, pR, J1);
        const double J1phi = (e.C1 > 0.0) ? J1 - e.C1 * J1r1 : J1;
        const double J1r1e1 = e.A1 * J1phi * p1 + e.B1 * J1phi + e.D1 * J1r1;
        const double p2 = f_downwind(pL, pR, J2);
        const double J2phi = (e.C2 > 0.0) ? J2 - e.C2 * J2r2 : J2;
        const double J2r2e2 = e.A2 * J2phi * p2 + e.B2 * J2phi + e.D2 * J2r2;
#pragma unroll
        for (int c = 0; c < D; ++c) F[2 + c] = -(Mf * ud[c]);
        F[M::IE1] = -(J1r1 * eK + J1r1e1);
        F[M::IE2] = -(J2r2 * eK + J2r2e2);
    }
}

// The Phase-Field face fluxes of model M (F stored negated; fnc the model's NCPF face terms).
template <class M, bool MIX>
__device__ __forceinline__ void pf_face_fluxes(double* F, double* fnc, const double* UL, const double* UR, double gq,
                                               const Eos& e, int phasic, int hll, unsigned int* err) {
    if constexpr (M::KIND == kModelSix) {
        pf_face_flux_six<M::D, MIX>(F, fnc, UL, UR, gq, e, phasic, hll, err);
    } else {
        pf_face_flux<M::D, MIX>(F, UL, UR, gq, e, phasic, hll, err);
        fnc[0] = 0.0;
    }
}

}  // namespace compas
