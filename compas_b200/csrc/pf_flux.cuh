// Phase-Field regularisation flux of one face (FIVEEQS, PhaseField.ID_Flux = 0 upwind/downwind,
// PhaseField.ID_FluxPhase2Flux = 1 mixture formulation) from the reconstructed face states and the
// face gradient of the regularisation potential Q.
//
// Reference:
//   FVM_Conservative2FluxPhaseField_K  include/Operators_Compressible5Eq_PhaseField/FVM_Conservative2FluxPhaseField_K_Compressible5Eq_PhaseField.H:15-69
//   FluxPhaseField                     include/Physics_Compressible5Eq_PhaseField/FluxPhaseField_Compressible5Eq_PhaseField.H
//   phase fluxes J_k rho_k, J_k (UD)   include/Physics_Compressible_TwoPhase_PhaseField/FluxPhasePhaseField_UD_Compressible_TwoPhase_PhaseField.H
//   mixture flux                       include/Physics_Compressible5Eq_PhaseField/FluxPhaseField_Mixture_Compressible5Eq_PhaseField.H
//   f_Upwind / f_Downwind              include/Operators_FV/f_Upwind.H, f_Downwind.H
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
                                             unsigned int* err) {
    using M = FiveEq<D>;
    constexpr int N = M::N;
    // phase fluxes (the two phases carry Q and -Q)
    const double g1 = gq, g2 = -g1;
    const double a1L = UL[M::IA], a1R = UR[M::IA];
    const double a2L = 1.0 - a1L, a2R = 1.0 - a1R;
    const double a2u = f_upwind(a2L, a2R, g1);
    const double a1u = f_upwind(a1L, a1R, g2);
    const double J1r1 = f_downwind(UL[0], UR[0], g1) * a2u * g1;
    const double J2r2 = f_downwind(UL[1], UR[1], g2) * a1u * g2;
    const double J1 = f_downwind(a1L, a1R, g1) * a2u * g1;
    const double J2 = f_downwind(a2L, a2R, g2) * a1u * g2;
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

}  // namespace compas
