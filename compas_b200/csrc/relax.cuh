// Instantaneous pressure relaxation of the six-equation model, applied after every RK stage.
//
// Closed form first (a quadratic for the relaxed pressure, then the volume fractions, then the
// pressure again from E1 + E2), kept wherever it is admissible; otherwise the safeguarded
// bracketed Newton/bisection solve of g(P) = sum_k alpha_k(P) - V on the active phases, and the
// phase energies reset at the common pressure. Operation order follows
//   include/Physics_Compressible6Eq/Relaxation_Pressure_Instantaneous_Compressible6Eq.H:32-220
//   include/RelaxationPressure_Safeguarded.H:17-256 (constants :76-84)
// so that the FP64 result is the reference's to the bit. Every loop is bounded (at most
// kMaxBracket + kMaxIter evaluations), so no input can make a thread spin.
#pragma once

#include "physics.cuh"

namespace compas {

constexpr double kRelaxRelTol = 1.0e-14;
constexpr double kRelaxResTol = 4.0e-15;
constexpr int kRelaxMaxIter = 100;
constexpr int kRelaxMaxBracket = 1100;
constexpr int kPathModel = 0, kPathSolve = 1, kPathOneActive = 2, kPathNoActive = 3, kPathNoRoot = 4;

__device__ __forceinline__ bool finite_d(double x) { return (x == x) && (fabs(x) <= DBL_MAX); }

// Safeguarded relaxation of NP phases (RelaxPressure_Safeguarded<N>): returns the path; AlphaR holds the
// relaxed volume fractions.
template <int NP>
__device__ __forceinline__ int relax_safeguarded(double* AlphaR, const double* Alpha, const double* Alpha_rho,
                                                const double* Phi, const double* Pi, const double* A,
                                                const double* B, double trace) {
    double c[NP], dd[NP], pinf[NP], shift[NP];
    bool active[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) shift[k] = 0.0;
    int n_active = 0;
    double pinf_m = DBL_MAX;
    for (int k = 0; k < NP; ++k) {
        const double gamma = (A[k] + 1.0) / A[k];
        pinf[k] = B[k] / (A[k] + 1.0);
        c[k] = (Pi[k] + Phi[k] * pinf[k]) / gamma;
        dd[k] = Phi[k] / gamma;
        active[k] = (Alpha[k] > 0.0) && (Alpha[k] > trace) && (Alpha_rho[k] > 0.0) && (c[k] > 0.0) &&
                    finite_d(c[k]) && finite_d(dd[k]);
        if (active[k]) {
            ++n_active;
            pinf_m = dmin(pinf_m, pinf[k]);
        }
    }
    double S_passive = 0.0;
    for (int k = 0; k < NP; ++k) {
        AlphaR[k] = Alpha[k];
        if (!active[k]) S_passive += Alpha[k];
    }
    const double V = 1.0 - S_passive;
    if (n_active == 0) return kPathNoActive;
    if (n_active == 1) {
        for (int k = 0; k < NP; ++k)
            if (active[k]) AlphaR[k] = V;
        return kPathOneActive;
    }
    double S = 0.0, Dsum = 0.0, S_Phi = 0.0, S_Pi = 0.0;
    for (int k = 0; k < NP; ++k) {
        if (active[k]) {
            S += Alpha[k];
            Dsum += dd[k];
            S_Phi += Phi[k];
            S_Pi += Pi[k];
            shift[k] = pinf[k] - pinf_m;
        }
    }
    const double g_inf = (S - V) - Dsum;
    if (!(g_inf < 0.0)) return kPathNoRoot;

    auto g = [&](double x) {
        double r = g_inf;
        for (int k = 0; k < NP; ++k)
            if (active[k]) r += c[k] / (x + shift[k]);
        return r;
    };
    auto g_scale = [&](double x) {
        double r = fabs(g_inf);
        for (int k = 0; k < NP; ++k)
            if (active[k]) r += c[k] / (x + shift[k]);
        return r;
    };
    auto dg = [&](double x) {
        double r = 0.0;
        for (int k = 0; k < NP; ++k)
            if (active[k]) {
                const double y = x + shift[k];
                r -= (c[k] / y) / y;
            }
        return r;
    };

    double x = (S_Phi > 0.0) ? S_Pi / S_Phi + pinf_m : -1.0;
    if (!(x > 0.0 && finite_d(x))) x = 1.0;
    double gx = g(x);
    double a = 0.0;
    double b = DBL_MAX;
    if (gx > 0.0) {
        a = x;
        for (int n = 0; n < kRelaxMaxBracket; ++n) {
            const double x4 = 4.0 * x;
            const double g4 = g(x4);
            if (!(g4 > 0.0)) {
                b = x4;
                break;
            }
            x = x4;
            gx = g4;
            a = x;
        }
    } else if (gx < 0.0) {
        b = x;
        for (int n = 0; n < kRelaxMaxBracket; ++n) {
            x *= 0.25;
            gx = g(x);
            if (gx > 0.0) {
                a = x;
                break;
            }
            b = x;
            if (!(gx < 0.0)) break;
        }
    }
    const bool bracketed = (gx == 0.0) || ((a > 0.0) && (b < DBL_MAX));
    if (!bracketed) return kPathNoRoot;
    if (gx != 0.0 && !(fabs(gx) <= kRelaxResTol * g_scale(x))) {
        for (int it = 0; it < kRelaxMaxIter; ++it) {
            double xn = x - gx / dg(x);
            if (!(xn > a && xn < b)) xn = (b > 16.0 * a) ? sqrt(a) * sqrt(b) : 0.5 * (a + b);
            const double step = fabs(xn - x);
            x = xn;
            gx = g(x);
            if (gx > 0.0)
                a = x;
            else if (gx < 0.0)
                b = x;
            else
                break;
            if (step <= kRelaxRelTol * x || fabs(gx) <= kRelaxResTol * g_scale(x)) break;
        }
    }
    for (int k = 0; k < NP; ++k)
        if (active[k]) AlphaR[k] = (Alpha[k] - dd[k]) + c[k] / (x + shift[k]);
    return kPathSolve;
}

// The two-phase instance (SixEq<D>).
__device__ __forceinline__ int relax_safeguarded2(double AlphaR[2], const double Alpha[2], const double Alpha_rho[2],
                                               const double Phi[2], const double Pi[2], const double A[2],
                                               const double B[2], double trace) {
    return relax_safeguarded<2>(AlphaR, Alpha, Alpha_rho, Phi, Pi, A, B, trace);
}

// Relax the state U of one cell in place (SixEq<D> layout). FAST (the mixed form): the same FP64
// root solve with the velocities and phase pressures of the entry state formed by multiplying with
// reciprocals (one division for 1/rho, the precomputed 1/A_k) and one reciprocal for the volume
// fraction normalisation, instead of the reference's divisions; the plain form (FAST = false) keeps
// the reference's operations to the bit.
template <int D, bool FAST = false>
__device__ __forceinline__ void relax_pressure(double* U, const Eos& e, double trace, unsigned int* err) {
    using M = SixEq<D>;
    constexpr int N = M::N;
    double W[N];
    if constexpr (FAST) {
        const double rho = U[0] + U[1];
        const double ir = 1.0 / rho;
        double u[3];
#pragma unroll
        for (int d = 0; d < D; ++d) u[d] = U[2 + d] * ir;
        const double k = ksum<D>(u);
        const double al1 = U[M::IA], al2 = 1.0 - al1;
        W[0] = U[0];
        W[1] = U[1];
#pragma unroll
        for (int d = 0; d < D; ++d) W[2 + d] = u[d];
        W[M::IA] = al1;
        const double e1 = U[M::IE1] - (0.5 * U[0]) * k;
        const double e2 = U[M::IE2] - (0.5 * U[1]) * k;
        if (e.C1 > 0.0) W[M::IE1] = M::phase_p(e1, al1, U[0], e.A1, e.B1, e.C1, e.D1, err);
        else W[M::IE1] = ((e1 - U[0] * e.D1) - al1 * e.B1) * e.iA1;
        if (e.C2 > 0.0) W[M::IE2] = M::phase_p(e2, al2, U[1], e.A2, e.B2, e.C2, e.D2, err);
        else W[M::IE2] = ((e2 - U[1] * e.D2) - al2 * e.B2) * e.iA2;
    } else {
        M::cons2prim(W, U, e, err);
    }
    const double a1r1 = W[0], a2r2 = W[1];
    const double alpha1 = W[M::IA];
    const double alpha2 = 1.0 - alpha1;
    const double a1p1 = W[M::IE1], a2p2 = W[M::IE2];
    const double A1 = e.A1, B1 = e.B1, A2 = e.A2, B2 = e.B2;
    double alpha1R, alpha2R, a1p1R, a2p2R;
    double Phi1_In = alpha1, Phi2_In = alpha2, Pi1_In = a1p1, Pi2_In = a2p2;
    bool raw_nan;
    double pQ;
    if (e.C1 > 0.0 || e.C2 > 0.0) {
        const double b1 = e.C1, b2 = e.C2;
        const double KE = 0.5 * ksum<D>(W + 2);
        const double E1 = (U[M::IE1] - a1r1 * KE) - a1r1 * e.D1;
        const double E2 = (U[M::IE2] - a2r2 * KE) - a2r2 * e.D2;
        const double Phi1 = alpha1 - b1 * a1r1;
        const double Phi2 = alpha2 - b2 * a2r2;
        const double Pi1 = (E1 - B1 * Phi1) / A1;
        const double Pi2 = (E2 - B2 * Phi2) / A2;
        Phi1_In = Phi1; Phi2_In = Phi2; Pi1_In = Pi1; Pi2_In = Pi2;
        const double aP = ((A1 * A2) * (Phi1 + Phi2) + A1 * Phi1) + A2 * Phi2;
        const double bP = (((A1 * B2) * Phi1 + (A2 * B1) * Phi2) - ((A2 + 1.0) * A1) * Pi1) - ((A1 + 1.0) * A2) * Pi2;
        const double cP = ((-B2) * A1) * Pi1 - (B1 * A2) * Pi2;
        double pR = (-bP + sqrt(bP * bP - (4.0 * aP) * cP)) / (2.0 * aP);
        pQ = pR;
        alpha1R = ((E1 + pR * alpha1) + (b1 * a1r1) * (A1 * pR + B1)) / ((A1 + 1.0) * pR + B1);
        alpha2R = ((E2 + pR * alpha2) + (b2 * a2r2) * (A2 * pR + B2)) / ((A2 + 1.0) * pR + B2);
        raw_nan = isnan(alpha1R) || isnan(alpha2R);
        if (isnan(alpha1R) && !isnan(alpha2R))
            alpha1R = 1.0 - alpha2R;
        else if (!isnan(alpha1R) && isnan(alpha2R))
            alpha2R = 1.0 - alpha1R;
        const double sum = alpha1R + alpha2R;
        alpha1R /= sum;
        alpha2R /= sum;
        const double Phi1R = nasg_xi(alpha1R, a1r1, b1, err) * alpha1R;
        const double Phi2R = nasg_xi(alpha2R, a2r2, b2, err) * alpha2R;
        pR = (((E1 + E2) - B1 * Phi1R) - B2 * Phi2R) / (A1 * Phi1R + A2 * Phi2R);
        a1p1R = alpha1R * pR;
        a2p2R = alpha2R * pR;
    } else {
        const double aP = ((A1 * A2) + A1 * alpha1) + A2 * alpha2;
        const double bP = (((A1 * B2) * alpha1 + (A2 * B1) * alpha2) - ((A2 + 1.0) * A1) * a1p1) - ((A1 + 1.0) * A2) * a2p2;
        const double cP = ((-B2) * A1) * a1p1 - (B1 * A2) * a2p2;
        double pR = (-bP + sqrt(bP * bP - (4.0 * aP) * cP)) / (2.0 * aP);
        pQ = pR;
        alpha1R = ((A1 * a1p1 + B1 * alpha1) + pR * alpha1) / ((A1 + 1.0) * pR + B1);
        alpha2R = ((A2 * a2p2 + B2 * alpha2) + pR * alpha2) / ((A2 + 1.0) * pR + B2);
        raw_nan = isnan(alpha1R) || isnan(alpha2R);
        if (isnan(alpha1R) && !isnan(alpha2R))
            alpha1R = 1.0 - alpha2R;
        else if (!isnan(alpha1R) && isnan(alpha2R))
            alpha2R = 1.0 - alpha1R;
        const double sum = alpha1R + alpha2R;
        if constexpr (FAST) {
            const double is = 1.0 / sum;
            alpha1R *= is;
            alpha2R *= is;
        } else {
            alpha1R /= sum;
            alpha2R /= sum;
        }
        pR = (((A1 * a1p1 + A2 * a2p2) + B1 * (alpha1 - alpha1R)) + B2 * (alpha2 - alpha2R)) /
             (A1 * alpha1R + A2 * alpha2R);
        a1p1R = alpha1R * pR;
        a2p2R = alpha2R * pR;
    }
    const double pinf_1 = e.pinf1;  // B1 / (A1 + 1), formed on the host with the same operation
    const double pinf_2 = e.pinf2;
    double pinf_m = DBL_MAX, pinf_scale = 0.0;
    if (alpha1 > 0.0) { pinf_m = dmin(pinf_m, pinf_1); pinf_scale = dmax(pinf_scale, fabs(pinf_1)); }
    if (alpha2 > 0.0) { pinf_m = dmin(pinf_m, pinf_2); pinf_scale = dmax(pinf_scale, fabs(pinf_2)); }
    const bool well = fabs(pQ + pinf_m) > 1.0e-8 * (fabs(pQ) + pinf_scale);
    const bool admissible = !raw_nan && well && finite_d(alpha1R) && finite_d(a1p1R) && finite_d(a2p2R) &&
                            !(alpha1 > 0.0 && alpha1 <= trace) && !(alpha2 > 0.0 && alpha2 <= trace);
    if (admissible) {
        W[M::IE1] = a1p1R;
        W[M::IE2] = a2p2R;
        W[M::IA] = alpha1R;
        if constexpr (FAST) {
            // the relaxation moves energy between the phases and leaves the momentum alone: keep the
            // entry momentum and total energy to the bit (the phase with the larger volume fraction takes
            // the remainder, as the safeguarded branch below does), so that the reciprocal-based entry
            // state does not make the total energy drift
            double mom[D];
#pragma unroll
            for (int d = 0; d < D; ++d) mom[d] = U[2 + d];
            const double E = U[M::IE1] + U[M::IE2];
            M::prim2cons(U, W, e, err);
#pragma unroll
            for (int d = 0; d < D; ++d) U[2 + d] = mom[d];
            if (alpha1R >= alpha2R)
                U[M::IE1] = E - U[M::IE2];
            else
                U[M::IE2] = E - U[M::IE1];
        } else {
            M::prim2cons(U, W, e, err);
        }
        return;
    }
    double AlphaR[2];
    const double Al[2] = {alpha1, alpha2}, Ar[2] = {a1r1, a2r2}, Ph[2] = {Phi1_In, Phi2_In}, Pi[2] = {Pi1_In, Pi2_In};
    const double Av[2] = {A1, A2}, Bv[2] = {B1, B2};
    const int path = relax_safeguarded2(AlphaR, Al, Ar, Ph, Pi, Av, Bv, trace);
    if (path == kPathNoRoot) flag_error(err, COMPAS_B200_ERR_RELAX_NOROOT);
    if (path != kPathSolve) AlphaR[0] = alpha1;
    AlphaR[1] = 1.0 - AlphaR[0];
    const double rho = a1r1 + a2r2;
    double rho_KE = 0.0;
    if (rho > 0.0) {
        double m2 = U[2] * U[2] + U[3] * U[3];
        if (D == 3) m2 = m2 + U[4] * U[4];
        rho_KE = (0.5 * m2) / rho;
    }
    const double KE = (rho > 0.0) ? rho_KE / rho : 0.0;
    const double E = U[M::IE1] + U[M::IE2];
    const double Phi1R = nasg_xi(AlphaR[0], a1r1, e.C1, err) * AlphaR[0];
    const double Phi2R = nasg_xi(AlphaR[1], a2r2, e.C2, err) * AlphaR[1];
    const double pR = (((((E - rho_KE) - a1r1 * e.D1) - a2r2 * e.D2) - B1 * Phi1R) - B2 * Phi2R) /
                      (A1 * Phi1R + A2 * Phi2R);
    double E1R = ((A1 * Phi1R) * pR + B1 * Phi1R) + a1r1 * (e.D1 + KE);
    double E2R = ((A2 * Phi2R) * pR + B2 * Phi2R) + a2r2 * (e.D2 + KE);
    if (AlphaR[0] >= AlphaR[1])
        E1R = E - E2R;
    else
        E2R = E - E1R;
    U[M::IE1] = E1R;
    U[M::IE2] = E2R;
    U[M::IA] = AlphaR[0];
}

}  // namespace compas
