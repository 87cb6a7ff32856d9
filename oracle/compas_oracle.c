/* Test infrastructure (oracle): plain-C restatement of the reference's finite-volume right-hand side
 * and TVD-RK3 level advance for the two-phase five- and six-equation models (WENO5 + HLLC, the
 * stiffened-gas / NASG EOS, the six-equation pressure relaxation) and the N-phase five-equation model
 * (FIVEEQS_NPHASE: WENO5 with the consistent limiter + HLLC). It follows the reference's own
 * per-face structure - every face converts its six stencil cells to primitives, reconstructs both
 * sides, converts back and calls the Riemann solver - with the same operations in the same order,
 * so that it agrees with the reference-header build (oracle/_ref) to the bit.
 *
 * Reference files followed (path:line in the reference tree):
 *   C2P / P2C / EOS 5Eq  include/Physics_Compressible5Eq/Conservative2Primitive_Compressible5Eq.H:15-61,
 *                        Primitive2Conservative_Compressible5Eq.H, EquationOfState_Mixture_Compressible5Eq.H:15-77
 *   C2P / P2C / EOS 6Eq  include/Physics_Compressible6Eq/Conservative2Primitive_Compressible6Eq.H:15-80,
 *                        Primitive2Conservative_Compressible6Eq.H, EquationOfState_Phase_Compressible6Eq.H:15-73
 *   NASG                 include/EquationOfState_NASG.H:26-58
 *   sound speeds         include/Physics_Compressible5Eq/SoundSpeed_Compressible5Eq.H, rho_c2_*_Compressible5Eq.H;
 *                        include/Physics_Compressible6Eq/SoundSpeed_Compressible6Eq.H, rho_c2_*_Compressible6Eq.H
 *   WENO5                include/Operators_FV/WENO5.H:12-75, Reconstruction2Face_WENO.H
 *   face reconstruction  include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_WENO5_D_Compressible5Eq.H,
 *                        FVM_Reconstruction2FaceLR_Conservative_WENO5_{D,K}_Compressible5Eq.H (6Eq alike)
 *   THINC                include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible5Eq.H:15-190,
 *                        include/Operators_Compressible6Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible6Eq.H:14-188,
 *                        include/Operators_FV/Reconstruction2Face_THINC_D.H, Reconstruction2Face_MUSCL_D.H, Limiter_Minmod.H,
 *                        include/Operators_FD/FDM_Normal_{X,Y,Z}FaceFromCenter_{K,D}.H, FDM_Gradient*FaceFromCenter_D.H
 *   HLLC                 include/Physics_Compressible5Eq/Riemann_HLLC_Compressible5Eq.H:16-194,
 *                        include/Physics_Compressible6Eq/Riemann_HLLC_Compressible6Eq.H:16-255
 *   face functor         include/Operators_Compressible5Eq/FVM_Conservative2FluxHyperbolic_K_Compressible5Eq.H:15-170,
 *                        include/Operators_Compressible6Eq/FVM_Conservative2FluxHyperbolic_K_Compressible6Eq.H:15-82
 *   divergence / NC      include/Operators_FV/FVM_SurfaceIntegral.H:17-28, FVM_Divergence_D.H,
 *                        include/Operators_Compressible5Eq/FVM_SurfaceIntegralNC_Compressible5Eq.H:15-52,
 *                        include/Operators_Compressible6Eq/FVM_SurfaceIntegralNC_Compressible6Eq.H:15-122
 *   N-phase model        include/Physics_Compressible5Eq_NPhase/{Conservative2Primitive,Primitive2Conservative,
 *                        EquationOfState_Mixture,SoundSpeed,rho_c2_Mixture,rho_c2_Phase,Conservative2Flux,
 *                        Riemann_HLLC,NonConservative}_Compressible5Eq_NPhase.H;
 *                        include/Operators_Compressible5Eq_NPhase/FVM_Reconstruction2Face_Conservative_WENO5_D_Compressible5Eq_NPhase.H,
 *                        FVM_Reconstruction2Face_Conservative_LimiterConsistent_Compressible5Eq_NPhase.H,
 *                        FVM_Reconstruction2Face_LimiterConsistent_Compressible5Eq_NPhase.H,
 *                        FVM_SurfaceIntegralNC_Compressible5Eq_NPhase.H; include/Operators_FV/Limiter_Consistent.H,
 *                        Reconstruction2Face_Linear.H
 *   relaxation           include/Physics_Compressible6Eq/Relaxation_Pressure_Instantaneous_Compressible6Eq.H:32-220,
 *                        include/RelaxationPressure_Safeguarded.H:17-256
 *   launch sites         source/Class_Compressible_PhaseField.cpp:3151-3391 (faces, divergence),
 *                        :3937-4107 (ThirdOrderSSPRK), :4472-4605 (EstTimeStep, CalculateInitialcmax);
 *                        source/COMPAS.cpp:2249-2303 (ComputeDt);
 *                        source/Class_Compressible6Eq_PhaseField.cpp:352-474 (BCs, Relaxation)
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_api.h"

#define MAXN 12
#define MAXP 4

typedef struct {
    int six, D, N, NC;
    int IE, IE1, IE2, IA; /* IE: 5Eq energy; IE1/IE2: 6Eq phase energies */
    int np;               /* FIVEEQS_NPHASE: phases (0 for the two-phase models) */
    int IM;               /* first momentum component */
    const cmp_case* c;
} Model;

static Model model_of(const cmp_case* c) {
    Model m;
    m.c = c;
    m.D = c->dim;
    m.six = (c->physics == 666);
    m.np = (c->physics == 55501) ? c->nphase : 0;
    if (m.np) {
        m.N = 2 * m.np + m.D + 1;
        m.NC = 1;
        m.IM = m.np;
        m.IE = m.np + m.D;
        m.IE1 = m.IE2 = m.IE;
        m.IA = m.np + m.D + 1;
        return m;
    }
    m.IM = 2;
    m.N = (m.six ? 5 : 4) + m.D;
    m.NC = m.six ? 3 : 1;
    m.IE = 2 + m.D;
    m.IE1 = 2 + m.D;
    m.IE2 = 3 + m.D;
    m.IA = m.six ? 4 + m.D : 3 + m.D;
    return m;
}

static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

static double nasg_phi(double alpha, double ar, double b) { return (b > 0.0) ? alpha - b * ar : alpha; }
static double nasg_xi(double alpha, double ar, double b) {
    return (b > 0.0 && alpha > 0.0) ? 1.0 - b * (ar / alpha) : 1.0;
}

static double ksum(const double* u, int D) {
    double s = u[0] * u[0] + u[1] * u[1];
    if (D == 3) s = s + u[2] * u[2];
    return s;
}

/* ---- N-phase five-equation model -------------------------------------------------------------- */
/* EquationOfState_Mixture sums over the phases, each from 0.0 */
static void np_sums(const Model* m, const double* ar, const double* al, double* rho_D, double* AP, double* BP) {
    const cmp_case* c = m->c;
    *rho_D = 0.0;
    for (int k = 0; k < m->np; ++k) *rho_D += ar[k] * c->Dk[k];
    *AP = 0.0;
    *BP = 0.0;
    for (int k = 0; k < m->np; ++k) {
        const double Phi = nasg_phi(al[k], ar[k], c->Ck[k]);
        *AP += Phi * c->Ak[k];
        *BP += Phi * c->Bk[k];
    }
}

static void np_c2p(const Model* m, const double* U, double* W) {
    const int D = m->D, NP = m->np;
    double rho = 0.0, u[3], rho_D, AP, BP;
    for (int k = 0; k < NP; ++k) rho += U[k];
    for (int d = 0; d < D; ++d) u[d] = U[m->IM + d] / rho;
    const double rho_e = U[m->IE] - (0.5) * rho * ksum(u, D);
    np_sums(m, U, U + m->IA, &rho_D, &AP, &BP);
    for (int k = 0; k < NP; ++k) {
        W[k] = U[k];
        W[m->IA + k] = U[m->IA + k];
    }
    for (int d = 0; d < D; ++d) W[m->IM + d] = u[d];
    W[m->IE] = (rho_e - rho_D - BP) / AP;
}

static void np_p2c(const Model* m, const double* W, double* U) {
    const int D = m->D, NP = m->np;
    double rho = 0.0, rho_D, AP, BP;
    for (int k = 0; k < NP; ++k) rho += W[k];
    np_sums(m, W, W + m->IA, &rho_D, &AP, &BP);
    const double rho_e = AP * W[m->IE] + BP + rho_D;
    for (int k = 0; k < NP; ++k) {
        U[k] = W[k];
        U[m->IA + k] = W[m->IA + k];
    }
    for (int d = 0; d < D; ++d) U[m->IM + d] = rho * W[m->IM + d];
    U[m->IE] = rho_e + (0.5) * rho * ksum(W + m->IM, D);
}

/* rho c^2 of the mixture from the phase values rhop_cp2 (rho_c2_Mixture) */
static double np_rho_c2(const Model* m, const double* W, const double* rc2, int id_k) {
    const cmp_case* c = m->c;
    if (id_k == 0) {
        double AP_rho_c2 = 0.0, AP = 0.0;
        for (int k = 0; k < m->np; ++k) {
            const double Phi = nasg_phi(W[m->IA + k], W[k], c->Ck[k]);
            AP_rho_c2 += W[m->IA + k] * c->Ak[k] * rc2[k];
            AP += Phi * c->Ak[k];
        }
        return AP_rho_c2 / AP;
    }
    double inv = 0.0;
    for (int k = 0; k < m->np; ++k) inv += nasg_phi(W[m->IA + k], W[k], c->Ck[k]) / rc2[k];
    return 1.0 / inv;
}

static void np_rc2_phases(const Model* m, double p, double* rc2) {
    const cmp_case* c = m->c;
    for (int k = 0; k < m->np; ++k) rc2[k] = ((c->Ak[k] + 1.0) * p + c->Bk[k]) / c->Ak[k];
}

static double np_sound_speed(const Model* m, const double* W) {
    double rc2[MAXP], rho = 0.0;
    np_rc2_phases(m, W[m->IE], rc2);
    const double rho_c2 = np_rho_c2(m, W, rc2, m->c->source_term);
    for (int k = 0; k < m->np; ++k) rho += W[k];
    return sqrt(rho_c2 / rho);
}

/* Limiter_Consistent (include/Operators_FV/Limiter_Consistent.H) */
static void np_limiter_consistent(int np, const double* slope, double* theta) {
    const double ep = 1.0e-10;
    double sum = 0.0, absv[MAXP];
    for (int k = 0; k < np; ++k) {
        sum += slope[k];
        absv[k] = fabs(slope[k]);
    }
    int imax = 0; /* std::max_element: the first largest */
    for (int k = 1; k < np; ++k)
        if (absv[imax] < absv[k]) imax = k;
    const double smax = slope[imax];
    if (fabs(smax) < ep || fabs(sum) < ep) {
        for (int k = 0; k < np; ++k) theta[k] = 1.0;
    } else {
        const double smaxS = smax - sum;
        for (int k = 0; k < np; ++k) theta[k] = dmax(dmin(smax / smaxS, 1.0), 0.0);
        theta[imax] = dmax(dmin(smaxS / smax, 1.0), 0.0);
    }
}

/* FVM_Reconstruction2Face_Conservative_LimiterConsistent: Uf in/out, Uc the stencil centre */
static void np_consistent(const Model* m, double* Uf, const double* Uc, double dx, int id_face) {
    const int NP = m->np;
    double Wf[MAXN], Wc[MAXN], s_ar[MAXP], s_al[MAXP], th[MAXP];
    np_c2p(m, Uf, Wf);
    np_c2p(m, Uc, Wc);
    for (int k = 0; k < NP; ++k) {
        s_ar[k] = (Wf[k] - Wc[k]) / ((double)id_face * 0.5 * dx);
        s_al[k] = (Wf[m->IA + k] - Wc[m->IA + k]) / ((double)id_face * 0.5 * dx);
    }
    np_limiter_consistent(NP, s_al, th);
    for (int k = 0; k < NP; ++k) {
        Wf[k] = Wc[k] + (double)id_face * 0.5 * (th[k] * s_ar[k]) * dx;
        Wf[m->IA + k] = Wc[m->IA + k] + (double)id_face * 0.5 * (th[k] * s_al[k]) * dx;
    }
    np_p2c(m, Wf, Uf);
}

/* ---- conversions ------------------------------------------------------------------------------ */
static void c2p(const Model* m, const double* U, double* W) {
    const cmp_case* c = m->c;
    const int D = m->D;
    if (m->np) {
        np_c2p(m, U, W);
        return;
    }
    double u[3];
    const double a1r1 = U[0], a2r2 = U[1], alpha1 = U[m->IA];
    const double rho = a1r1 + a2r2;
    for (int d = 0; d < D; ++d) u[d] = U[2 + d] / rho;
    W[0] = a1r1;
    W[1] = a2r2;
    for (int d = 0; d < D; ++d) W[2 + d] = u[d];
    W[m->IA] = alpha1;
    if (!m->six) {
        const double rho_e = U[m->IE] - (0.5 * rho) * ksum(u, D);
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = nasg_phi(alpha1, a1r1, c->C1), phi2 = nasg_phi(alpha2, a2r2, c->C2);
        const double rho_D = a1r1 * c->D1 + a2r2 * c->D2;
        const double AP = phi1 * c->A1 + phi2 * c->A2;
        const double BP = phi1 * c->B1 + phi2 * c->B2;
        W[m->IE] = ((rho_e - rho_D) - BP) / AP;
    } else {
        const double alpha2 = 1.0 - alpha1;
        const double k = ksum(u, D);
        const double e1 = U[m->IE1] - (0.5 * a1r1) * k;
        const double e2 = U[m->IE2] - (0.5 * a2r2) * k;
        const double xi1 = nasg_xi(alpha1, a1r1, c->C1), xi2 = nasg_xi(alpha2, a2r2, c->C2);
        W[m->IE1] = ((e1 - a1r1 * c->D1) - (xi1 * alpha1) * c->B1) / (c->A1 * xi1);
        W[m->IE2] = ((e2 - a2r2 * c->D2) - (xi2 * alpha2) * c->B2) / (c->A2 * xi2);
    }
}

static void p2c(const Model* m, const double* W, double* U) {
    const cmp_case* c = m->c;
    const int D = m->D;
    if (m->np) {
        np_p2c(m, W, U);
        return;
    }
    const double a1r1 = W[0], a2r2 = W[1], alpha1 = W[m->IA];
    const double alpha2 = 1.0 - alpha1;
    const double rho = a1r1 + a2r2;
    U[0] = a1r1;
    U[1] = a2r2;
    for (int d = 0; d < D; ++d) U[2 + d] = rho * W[2 + d];
    U[m->IA] = alpha1;
    if (!m->six) {
        const double phi1 = nasg_phi(alpha1, a1r1, c->C1), phi2 = nasg_phi(alpha2, a2r2, c->C2);
        const double rho_D = a1r1 * c->D1 + a2r2 * c->D2;
        const double AP = phi1 * c->A1 + phi2 * c->A2;
        const double BP = phi1 * c->B1 + phi2 * c->B2;
        const double rho_e = (AP * W[m->IE] + BP) + rho_D;
        U[m->IE] = rho_e + (0.5 * rho) * ksum(W + 2, D);
    } else {
        const double xi1 = nasg_xi(alpha1, a1r1, c->C1), xi2 = nasg_xi(alpha2, a2r2, c->C2);
        const double e1 = ((c->A1 * xi1) * W[m->IE1] + (xi1 * alpha1) * c->B1) + a1r1 * c->D1;
        const double e2 = ((c->A2 * xi2) * W[m->IE2] + (xi2 * alpha2) * c->B2) + a2r2 * c->D2;
        const double k = ksum(W + 2, D);
        U[m->IE1] = e1 + (0.5 * a1r1) * k;
        U[m->IE2] = e2 + (0.5 * a2r2) * k;
    }
}

static double sound_speed(const Model* m, const double* W) {
    const cmp_case* c = m->c;
    if (m->np) return np_sound_speed(m, W);
    const double a1r1 = W[0], a2r2 = W[1], alpha1 = W[m->IA];
    double rho_c2;
    if (!m->six) {
        const double p = W[m->IE];
        const double r1 = ((c->A1 + 1.0) * p + c->B1) / c->A1;
        const double r2 = ((c->A2 + 1.0) * p + c->B2) / c->A2;
        const double alpha2 = 1.0 - alpha1;
        const double phi1 = nasg_phi(alpha1, a1r1, c->C1), phi2 = nasg_phi(alpha2, a2r2, c->C2);
        if (c->source_term == 0) {
            const double num = (alpha1 * c->A1) * r1 + (alpha2 * c->A2) * r2;
            rho_c2 = num / (phi1 * c->A1 + phi2 * c->A2);
        } else {
            rho_c2 = 1.0 / (phi1 / r1 + phi2 / r2);
        }
    } else {
        const double xi1 = nasg_xi(alpha1, a1r1, c->C1), xi2 = nasg_xi(1.0 - alpha1, a2r2, c->C2);
        const double r1 = ((c->A1 + 1.0) * W[m->IE1] + alpha1 * c->B1) / (c->A1 * xi1);
        const double r2 = ((c->A2 + 1.0) * W[m->IE2] + (1.0 - alpha1) * c->B2) / (c->A2 * xi2);
        rho_c2 = r1 + r2;
    }
    return sqrt(rho_c2 / (a1r1 + a2r2));
}

static void phys_flux(const Model* m, const double* U, const double* W, int d, double* F) {
    if (m->np) {
        const double V = W[m->IM + d], p = W[m->IE];
        for (int k = 0; k < m->np; ++k) {
            F[k] = U[k] * V;
            F[m->IA + k] = U[m->IA + k] * V;
        }
        for (int k = 0; k < m->D; ++k) F[m->IM + k] = U[m->IM + k] * V;
        F[m->IE] = (U[m->IE] + p) * V;
        F[m->IM + d] += p;
        return;
    }
    const double V = W[2 + d];
    F[0] = U[0] * V;
    F[1] = U[1] * V;
    for (int k = 0; k < m->D; ++k) F[2 + k] = U[2 + k] * V;
    F[m->IA] = U[m->IA] * V;
    if (!m->six) {
        F[m->IE] = (U[m->IE] + W[m->IE]) * V;
        F[2 + d] = F[2 + d] + W[m->IE];
    } else {
        F[m->IE1] = (U[m->IE1] + W[m->IE1]) * V;
        F[m->IE2] = (U[m->IE2] + W[m->IE2]) * V;
        F[2 + d] = F[2 + d] + (W[m->IE1] + W[m->IE2]);
    }
}

/* ---- WENO5 -------------------------------------------------------------------------------------- */
static double weno5(double f_mm, double f_m, double f_c, double f_p, double f_pp, int side) {
    double q0, q1, q2, d0, d2;
    if (side == 1) {
        q0 = f_c + (2.0 / 3.0) * (f_p - f_c) - (1.0 / 6.0) * (f_pp - f_p);
        q1 = f_c + (1.0 / 6.0) * (f_c - f_m) + (1.0 / 3.0) * (f_p - f_c);
        q2 = f_c - (1.0 / 3.0) * (f_m - f_mm) + (5.0 / 6.0) * (f_c - f_m);
        d0 = 3.0 / 10.0;
        d2 = 1.0 / 10.0;
    } else {
        q0 = f_c - (5.0 / 6.0) * (f_p - f_c) + (1.0 / 3.0) * (f_pp - f_p);
        q1 = f_c - (1.0 / 3.0) * (f_c - f_m) - (1.0 / 6.0) * (f_p - f_c);
        q2 = f_c + (1.0 / 6.0) * (f_m - f_mm) - (2.0 / 3.0) * (f_c - f_m);
        d0 = 1.0 / 10.0;
        d2 = 3.0 / 10.0;
    }
    const double d1 = 1.0 - d0 - d2;
    const double IS0 = (10.0 / 3.0) * (f_p - f_c) * (f_p - f_c) - (11.0 / 3.0) * (f_p - f_c) * (f_pp - f_p) +
                       (4.0 / 3.0) * (f_pp - f_p) * (f_pp - f_p);
    const double IS1 = -(5.0 / 3.0) * (f_c - f_m) * (f_p - f_c) + (4.0 / 3.0) * (f_c - f_m) * (f_c - f_m) +
                       (4.0 / 3.0) * (f_p - f_c) * (f_p - f_c);
    const double IS2 = (10.0 / 3.0) * (f_c - f_m) * (f_c - f_m) - (11.0 / 3.0) * (f_m - f_mm) * (f_c - f_m) +
                       (4.0 / 3.0) * (f_m - f_mm) * (f_m - f_mm);
    double IS01 = IS0 / IS1;
    if (isnan(IS01)) IS01 = 1.0;
    const double IS10 = 1.0 / IS01;
    double IS02 = IS0 / IS2;
    if (isnan(IS02)) IS02 = 1.0;
    const double IS20 = 1.0 / IS02;
    double IS12 = IS1 / IS2;
    if (isnan(IS12)) IS12 = 1.0;
    const double IS21 = 1.0 / IS12;
    const double w0 = d0 / (d0 + (IS01 * IS01) * d1 + (IS02 * IS02) * d2);
    const double w1 = d1 / ((IS10 * IS10) * d0 + d1 + (IS12 * IS12) * d2);
    const double w2 = d2 / ((IS20 * IS20) * d0 + (IS21 * IS21) * d1 + d2);
    double f = 0.0;
    f += w0 * q0;
    f += w1 * q1;
    f += w2 * q2;
    return f;
}

/* WENO5 candidates q and weights w (w may be NULL) */
static void weno5_parts(double f_mm, double f_m, double f_c, double f_p, double f_pp, int side, double* q, double* w) {
    double d0, d2;
    if (side == 1) {
        q[0] = f_c + (2.0 / 3.0) * (f_p - f_c) - (1.0 / 6.0) * (f_pp - f_p);
        q[1] = f_c + (1.0 / 6.0) * (f_c - f_m) + (1.0 / 3.0) * (f_p - f_c);
        q[2] = f_c - (1.0 / 3.0) * (f_m - f_mm) + (5.0 / 6.0) * (f_c - f_m);
        d0 = 3.0 / 10.0;
        d2 = 1.0 / 10.0;
    } else {
        q[0] = f_c - (5.0 / 6.0) * (f_p - f_c) + (1.0 / 3.0) * (f_pp - f_p);
        q[1] = f_c - (1.0 / 3.0) * (f_c - f_m) - (1.0 / 6.0) * (f_p - f_c);
        q[2] = f_c + (1.0 / 6.0) * (f_m - f_mm) - (2.0 / 3.0) * (f_c - f_m);
        d0 = 1.0 / 10.0;
        d2 = 3.0 / 10.0;
    }
    if (!w) return;
    const double d1 = 1.0 - d0 - d2;
    const double IS0 = (10.0 / 3.0) * (f_p - f_c) * (f_p - f_c) - (11.0 / 3.0) * (f_p - f_c) * (f_pp - f_p) +
                       (4.0 / 3.0) * (f_pp - f_p) * (f_pp - f_p);
    const double IS1 = -(5.0 / 3.0) * (f_c - f_m) * (f_p - f_c) + (4.0 / 3.0) * (f_c - f_m) * (f_c - f_m) +
                       (4.0 / 3.0) * (f_p - f_c) * (f_p - f_c);
    const double IS2 = (10.0 / 3.0) * (f_c - f_m) * (f_c - f_m) - (11.0 / 3.0) * (f_m - f_mm) * (f_c - f_m) +
                       (4.0 / 3.0) * (f_m - f_mm) * (f_m - f_mm);
    double IS01 = IS0 / IS1;
    if (isnan(IS01)) IS01 = 1.0;
    const double IS10 = 1.0 / IS01;
    double IS02 = IS0 / IS2;
    if (isnan(IS02)) IS02 = 1.0;
    const double IS20 = 1.0 / IS02;
    double IS12 = IS1 / IS2;
    if (isnan(IS12)) IS12 = 1.0;
    const double IS21 = 1.0 / IS12;
    w[0] = d0 / (d0 + (IS01 * IS01) * d1 + (IS02 * IS02) * d2);
    w[1] = d1 / ((IS10 * IS10) * d0 + d1 + (IS12 * IS12) * d2);
    w[2] = d2 / ((IS20 * IS20) * d0 + (IS21 * IS21) * d1 + d2);
}

static double wsum(const double* q, const double* w) {
    double f = 0.0;
    for (int i = 0; i < 3; ++i) f += w[i] * q[i];
    return f;
}

/* Limiter_Bound, ID_BoundType -1, f_min 0, Weight 1/12 (include/Operators_FV/Limiter_Bound.H,
 * Limiter_BoundMin.H, fC_QuadratureRule.H) */
static double theta_min0(double f_c, double fL, double fR) {
    const double Wt = 1.0 / 12.0;
    const double fC = (f_c - Wt * fL - Wt * fR) / (1.0 - 2.0 * Wt);
    double mn = fC;
    if (fL < mn) mn = fL;
    if (fR < mn) mn = fR;
    return dmin(1.0, dmax(0.0, f_c - 0.0) / dmax(0.0, f_c - mn));
}

/* WENO5B masses and volume fraction of the cell at P[2] (P: primitive stencil of 5 cells) at face side
 * (include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_WENO5B_D_Compressible5Eq.H:15-320) */
static void weno5b_bounded(const Model* m, double P[][MAXN], int side, double* WF) {
    double Ar[2][5], Al[2][5], rL[2], rR[2], aL[2], aR[2], q[3], w[3], qa[3];
    for (int s = 0; s < 5; ++s) {
        Ar[0][s] = P[s][0];
        Ar[1][s] = P[s][1];
        Al[0][s] = P[s][m->IA];
        Al[1][s] = 1.0 - P[s][m->IA];
    }
    const double inf_unused = 0.0;
    (void)inf_unused;
    double sumL = 0.0, sumR = 0.0;
    for (int k = 0; k < 2; ++k) {
        const double* fr = Ar[k];
        const double* fa = Al[k];
        weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], 1, q, w);
        rL[k] = wsum(q, w);
        weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], 1, qa, NULL);
        aL[k] = wsum(qa, w);
        weno5_parts(fr[0], fr[1], fr[2], fr[3], fr[4], -1, q, w);
        rR[k] = wsum(q, w);
        weno5_parts(fa[0], fa[1], fa[2], fa[3], fa[4], -1, qa, NULL);
        aR[k] = wsum(qa, w);
        const double th = dmin(theta_min0(fr[2], rL[k], rR[k]), theta_min0(fa[2], aL[k], aR[k]));
        rL[k] = fr[2] + th * (rL[k] - fr[2]);
        aL[k] = fa[2] + th * (aL[k] - fa[2]);
        rR[k] = fr[2] + th * (rR[k] - fr[2]);
        aR[k] = fa[2] + th * (aR[k] - fa[2]);
        sumL += aL[k];
        sumR += aR[k];
    }
    double Th = 1.0;
    for (int k = 0; k < 2; ++k) {
        rL[k] /= sumL;
        aL[k] /= sumL;
        rR[k] /= sumR;
        aR[k] /= sumR;
        const double tr = theta_min0(Ar[k][2], rL[k], rR[k]);
        const double ta = theta_min0(Al[k][2], aL[k], aR[k]);
        if (tr < Th) Th = tr;
        if (ta < Th) Th = ta;
    }
    WF[0] = Ar[0][2] + Th * ((side == 1 ? rL[0] : rR[0]) - Ar[0][2]);
    WF[1] = Ar[1][2] + Th * ((side == 1 ? rL[1] : rR[1]) - Ar[1][2]);
    WF[m->IA] = Al[0][2] + Th * ((side == 1 ? aL[0] : aR[0]) - Al[0][2]);
}

/* ---- Riemann solver ------------------------------------------------------------------------------ */
static void hllc(const Model* m, const double* UL, const double* UR, int d, double* Fo, double* fnc, double* cmax) {
    const int N = m->N, D = m->D;
    double WL[MAXN], WR[MAXN], FL[MAXN], FR[MAXN];
    c2p(m, UL, WL);
    c2p(m, UR, WR);
    phys_flux(m, UL, WL, d, FL);
    phys_flux(m, UR, WR, d, FR);
    const double cL = sound_speed(m, WL), cR = sound_speed(m, WR);
    const double VL = WL[m->IM + d], VR = WR[m->IM + d];
    double rhoL = WL[0] + WL[1], rhoR = WR[0] + WR[1];
    if (m->np) {
        rhoL = 0.0;
        rhoR = 0.0;
        for (int k = 0; k < m->np; ++k) {
            rhoL += WL[k];
            rhoR += WR[k];
        }
    }
    double SL, SR, pL, pR;
    if (!m->six) {
        pL = WL[m->IE];
        pR = WR[m->IE];
        const double V_avg = 0.5 * (VL + VR), c_avg = 0.5 * (cL + cR);
        SL = dmin(V_avg - c_avg, VL - cL);
        SR = dmax(V_avg + c_avg, VR + cR);
    } else {
        pL = WL[m->IE1] + WL[m->IE2];
        pR = WR[m->IE1] + WR[m->IE2];
        SL = dmin(VL - cL, VR - cR);
        SR = dmax(VL + cL, VR + cR);
    }
    const double Sm = dmin(0.0, SL), Sp = dmax(0.0, SR);
    const double S = (pR - pL + rhoL * VL * (SL - VL) - rhoR * VR * (SR - VR)) / (rhoL * (SL - VL) - rhoR * (SR - VR));
    const double s = sgn(S);
    double UsL[MAXN], UsR[MAXN];
    if (!m->six) {
        for (int i = 0; i < N; ++i) {
            UsL[i] = (SL - VL) / (SL - S) * UL[i];
            UsR[i] = (SR - VR) / (SR - S) * UR[i];
            if (i == m->IM + d) {
                UsL[i] += (SL - VL) / (SL - S) * rhoL * (S - VL);
                UsR[i] += (SR - VR) / (SR - S) * rhoR * (S - VR);
            } else if (i == m->IE) {
                UsL[i] += (SL - VL) / (SL - S) * (S - VL) * (rhoL * S + pL / (SL - VL));
                UsR[i] += (SR - VR) / (SR - S) * (S - VR) * (rhoR * S + pR / (SR - VR));
            }
        }
        double vel = 0.5 * (1.0 + s) * WL[m->IM + d] + 0.5 * (1.0 - s) * WR[m->IM + d];
        vel += 0.5 * (1.0 + s) * Sm * ((SL - VL) / (SL - S) - 1.0) + 0.5 * (1.0 - s) * Sp * ((SR - VR) / (SR - S) - 1.0);
        fnc[0] = vel;
    } else {
        const double a1r1L = WL[0], a2r2L = WL[1], a1r1R = WR[0], a2r2R = WR[1];
        const double a1p1L = WL[m->IE1], a2p2L = WL[m->IE2], a1p1R = WR[m->IE1], a2p2R = WR[m->IE2];
        const double a1r1Ls = (SL - VL) / (SL - S) * a1r1L, a1r1Rs = (SR - VR) / (SR - S) * a1r1R;
        const double a2r2Ls = (SL - VL) / (SL - S) * a2r2L, a2r2Rs = (SR - VR) / (SR - S) * a2r2R;
        UsL[0] = a1r1Ls; UsL[1] = a2r2Ls; UsR[0] = a1r1Rs; UsR[1] = a2r2Rs;
        for (int k = 0; k < D; ++k) {
            UsL[2 + k] = (SL - VL) / (SL - S) * rhoL * (WL[2 + k] + (double)(d == k) * (S - WL[2 + k]));
            UsR[2 + k] = (SR - VR) / (SR - S) * rhoR * (WR[2 + k] + (double)(d == k) * (S - WR[2 + k]));
        }
        const double a1p1Ls = a1p1L + (VL - SL) * a1r1L * VL - (S - SL) * a1r1Ls * S;
        const double a1p1Rs = a1p1R + (VR - SR) * a1r1R * VR - (S - SR) * a1r1Rs * S;
        const double a2p2Ls = a2p2L + (VL - SL) * a2r2L * VL - (S - SL) * a2r2Ls * S;
        const double a2p2Rs = a2p2R + (VR - SR) * a2r2R * VR - (S - SR) * a2r2Rs * S;
        UsL[m->IE1] = ((VL - SL) * UL[m->IE1] + VL * a1p1L - S * a1p1Ls) / (S - SL);
        UsR[m->IE1] = ((VR - SR) * UR[m->IE1] + VR * a1p1R - S * a1p1Rs) / (S - SR);
        UsL[m->IE2] = ((VL - SL) * UL[m->IE2] + VL * a2p2L - S * a2p2Ls) / (S - SL);
        UsR[m->IE2] = ((VR - SR) * UR[m->IE2] + VR * a2p2R - S * a2p2Rs) / (S - SR);
        UsL[m->IA] = (SL - VL) / (SL - S) * WL[m->IA];
        UsR[m->IA] = (SR - VR) / (SR - S) * WR[m->IA];
        const double uLd = WL[2 + d], uRd = WR[2 + d];
        double vel = 0.5 * (1.0 + s) * uLd + 0.5 * (1.0 - s) * uRd;
        vel += 0.5 * (1.0 + s) * Sm * ((SL - VL) / (SL - S) - 1.0) + 0.5 * (1.0 - s) * Sp * ((SR - VR) / (SR - S) - 1.0);
        fnc[0] = vel;
        fnc[1] = 0.5 * (1.0 + s) * (uLd * a1p1L + 1.0 * Sm * (VL * a1p1L - S * a1p1Ls) / (S - SL)) +
                 0.5 * (1.0 - s) * (uRd * a1p1R + 1.0 * Sp * (VR * a1p1R - S * a1p1Rs) / (S - SR));
        fnc[2] = 0.5 * (1.0 + s) * (uLd * a2p2L + 1.0 * Sm * (VL * a2p2L - S * a2p2Ls) / (S - SL)) +
                 0.5 * (1.0 - s) * (uRd * a2p2R + 1.0 * Sp * (VR * a2p2R - S * a2p2Rs) / (S - SR));
    }
    for (int i = 0; i < N; ++i)
        Fo[i] = 0.5 * (1.0 + s) * (FL[i] + Sm * (UsL[i] - UL[i])) + 0.5 * (1.0 - s) * (FR[i] + Sp * (UsR[i] - UR[i]));
    *cmax = dmax(cL + sqrt(ksum(WL + m->IM, D)), cR + sqrt(ksum(WR + m->IM, D)));
}

/* ---- six-equation pressure relaxation -------------------------------------------------------------- */
static int finite_d(double x) { return (x == x) && (fabs(x) <= DBL_MAX); }

static int relax_safeguarded2(double* AlphaR, const double* Alpha, const double* Ar, const double* Phi,
                              const double* Pi, const double* A, const double* B, double trace) {
    double c[2], dd[2], pinf[2], shift[2] = {0.0, 0.0};
    int active[2], n_active = 0;
    double pinf_m = DBL_MAX;
    for (int k = 0; k < 2; ++k) {
        const double gamma = (A[k] + 1.0) / A[k];
        pinf[k] = B[k] / (A[k] + 1.0);
        c[k] = (Pi[k] + Phi[k] * pinf[k]) / gamma;
        dd[k] = Phi[k] / gamma;
        active[k] = (Alpha[k] > 0.0) && (Alpha[k] > trace) && (Ar[k] > 0.0) && (c[k] > 0.0) && finite_d(c[k]) &&
                    finite_d(dd[k]);
        if (active[k]) {
            ++n_active;
            pinf_m = dmin(pinf_m, pinf[k]);
        }
    }
    double S_passive = 0.0;
    for (int k = 0; k < 2; ++k) {
        AlphaR[k] = Alpha[k];
        if (!active[k]) S_passive += Alpha[k];
    }
    const double V = 1.0 - S_passive;
    if (n_active == 0) return 3;
    if (n_active == 1) {
        for (int k = 0; k < 2; ++k)
            if (active[k]) AlphaR[k] = V;
        return 2;
    }
    double S = 0.0, Ds = 0.0, S_Phi = 0.0, S_Pi = 0.0;
    for (int k = 0; k < 2; ++k)
        if (active[k]) {
            S += Alpha[k];
            Ds += dd[k];
            S_Phi += Phi[k];
            S_Pi += Pi[k];
            shift[k] = pinf[k] - pinf_m;
        }
    const double g_inf = (S - V) - Ds;
    if (!(g_inf < 0.0)) return 4;
#define G_OF(xx, out)                                                      \
    do {                                                                   \
        double r_ = g_inf;                                                 \
        for (int k_ = 0; k_ < 2; ++k_)                                     \
            if (active[k_]) r_ += c[k_] / ((xx) + shift[k_]);              \
        (out) = r_;                                                        \
    } while (0)
#define GS_OF(xx, out)                                                     \
    do {                                                                   \
        double r_ = fabs(g_inf);                                           \
        for (int k_ = 0; k_ < 2; ++k_)                                     \
            if (active[k_]) r_ += c[k_] / ((xx) + shift[k_]);              \
        (out) = r_;                                                        \
    } while (0)
    double x = (S_Phi > 0.0) ? S_Pi / S_Phi + pinf_m : -1.0;
    if (!(x > 0.0 && finite_d(x))) x = 1.0;
    double gx, a = 0.0, b = DBL_MAX;
    G_OF(x, gx);
    if (gx > 0.0) {
        a = x;
        for (int n = 0; n < 1100; ++n) {
            const double x4 = 4.0 * x;
            double g4;
            G_OF(x4, g4);
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
        for (int n = 0; n < 1100; ++n) {
            x *= 0.25;
            G_OF(x, gx);
            if (gx > 0.0) {
                a = x;
                break;
            }
            b = x;
            if (!(gx < 0.0)) break;
        }
    }
    const int bracketed = (gx == 0.0) || ((a > 0.0) && (b < DBL_MAX));
    if (!bracketed) return 4;
    double gsc;
    GS_OF(x, gsc);
    if (gx != 0.0 && !(fabs(gx) <= 4.0e-15 * gsc)) {
        for (int it = 0; it < 100; ++it) {
            double dg = 0.0;
            for (int k = 0; k < 2; ++k)
                if (active[k]) {
                    const double y = x + shift[k];
                    dg -= (c[k] / y) / y;
                }
            double xn = x - gx / dg;
            if (!(xn > a && xn < b)) xn = (b > 16.0 * a) ? sqrt(a) * sqrt(b) : 0.5 * (a + b);
            const double step = fabs(xn - x);
            x = xn;
            G_OF(x, gx);
            if (gx > 0.0)
                a = x;
            else if (gx < 0.0)
                b = x;
            else
                break;
            GS_OF(x, gsc);
            if (step <= 1.0e-14 * x || fabs(gx) <= 4.0e-15 * gsc) break;
        }
    }
#undef G_OF
#undef GS_OF
    for (int k = 0; k < 2; ++k)
        if (active[k]) AlphaR[k] = Alpha[k] - dd[k] + c[k] / (x + shift[k]);
    return 1;
}

static void relax_cell(const Model* m, const double* U, double* UR) {
    const cmp_case* c = m->c;
    const int N = m->N, D = m->D;
    double W[MAXN];
    c2p(m, U, W);
    const double a1r1 = W[0], a2r2 = W[1], alpha1 = W[m->IA], alpha2 = 1.0 - alpha1;
    const double a1p1 = W[m->IE1], a2p2 = W[m->IE2];
    const double A1 = c->A1, B1 = c->B1, A2 = c->A2, B2 = c->B2;
    double alpha1R, alpha2R, a1p1R, a2p2R, pQ;
    double Phi1_In = alpha1, Phi2_In = alpha2, Pi1_In = a1p1, Pi2_In = a2p2;
    int raw_nan;
    if (c->C1 > 0.0 || c->C2 > 0.0) {
        const double b1 = c->C1, b2 = c->C2;
        const double KE = 0.5 * ksum(W + 2, D);
        const double E1 = U[m->IE1] - a1r1 * KE - a1r1 * c->D1;
        const double E2 = U[m->IE2] - a2r2 * KE - a2r2 * c->D2;
        const double Phi1 = alpha1 - b1 * a1r1, Phi2 = alpha2 - b2 * a2r2;
        const double Pi1 = (E1 - B1 * Phi1) / A1, Pi2 = (E2 - B2 * Phi2) / A2;
        Phi1_In = Phi1; Phi2_In = Phi2; Pi1_In = Pi1; Pi2_In = Pi2;
        const double aP = A1 * A2 * (Phi1 + Phi2) + A1 * Phi1 + A2 * Phi2;
        const double bP = A1 * B2 * Phi1 + A2 * B1 * Phi2 - (A2 + 1.0) * A1 * Pi1 - (A1 + 1.0) * A2 * Pi2;
        const double cP = -B2 * A1 * Pi1 - B1 * A2 * Pi2;
        double pR = (-bP + sqrt(bP * bP - 4.0 * aP * cP)) / (2.0 * aP);
        pQ = pR;
        alpha1R = (E1 + pR * alpha1 + b1 * a1r1 * (A1 * pR + B1)) / ((A1 + 1.0) * pR + B1);
        alpha2R = (E2 + pR * alpha2 + b2 * a2r2 * (A2 * pR + B2)) / ((A2 + 1.0) * pR + B2);
        raw_nan = isnan(alpha1R) || isnan(alpha2R);
        if (isnan(alpha1R) && !isnan(alpha2R)) alpha1R = 1.0 - alpha2R;
        else if (!isnan(alpha1R) && isnan(alpha2R)) alpha2R = 1.0 - alpha1R;
        const double sum = alpha1R + alpha2R;
        alpha1R /= sum;
        alpha2R /= sum;
        const double Phi1R = nasg_xi(alpha1R, a1r1, b1) * alpha1R;
        const double Phi2R = nasg_xi(alpha2R, a2r2, b2) * alpha2R;
        pR = (E1 + E2 - B1 * Phi1R - B2 * Phi2R) / (A1 * Phi1R + A2 * Phi2R);
        a1p1R = alpha1R * pR;
        a2p2R = alpha2R * pR;
    } else {
        const double aP = A1 * A2 + A1 * alpha1 + A2 * alpha2;
        const double bP = A1 * B2 * alpha1 + A2 * B1 * alpha2 - (A2 + 1.0) * A1 * a1p1 - (A1 + 1.0) * A2 * a2p2;
        const double cP = -B2 * A1 * a1p1 - B1 * A2 * a2p2;
        double pR = (-bP + sqrt(bP * bP - 4.0 * aP * cP)) / (2.0 * aP);
        pQ = pR;
        alpha1R = (A1 * a1p1 + B1 * alpha1 + pR * alpha1) / ((A1 + 1.0) * pR + B1);
        alpha2R = (A2 * a2p2 + B2 * alpha2 + pR * alpha2) / ((A2 + 1.0) * pR + B2);
        raw_nan = isnan(alpha1R) || isnan(alpha2R);
        if (isnan(alpha1R) && !isnan(alpha2R)) alpha1R = 1.0 - alpha2R;
        else if (!isnan(alpha1R) && isnan(alpha2R)) alpha2R = 1.0 - alpha1R;
        const double sum = alpha1R + alpha2R;
        alpha1R /= sum;
        alpha2R /= sum;
        pR = (A1 * a1p1 + A2 * a2p2 + B1 * (alpha1 - alpha1R) + B2 * (alpha2 - alpha2R)) / (A1 * alpha1R + A2 * alpha2R);
        a1p1R = alpha1R * pR;
        a2p2R = alpha2R * pR;
    }
    const double pinf_1 = B1 / (A1 + 1.0), pinf_2 = B2 / (A2 + 1.0);
    double pinf_m = DBL_MAX, pinf_scale = 0.0;
    if (alpha1 > 0.0) { pinf_m = dmin(pinf_m, pinf_1); pinf_scale = dmax(pinf_scale, fabs(pinf_1)); }
    if (alpha2 > 0.0) { pinf_m = dmin(pinf_m, pinf_2); pinf_scale = dmax(pinf_scale, fabs(pinf_2)); }
    const int well = fabs(pQ + pinf_m) > 1.0e-8 * (fabs(pQ) + pinf_scale);
    const double tr = c->relax_trace;
    const int admissible = !raw_nan && well && finite_d(alpha1R) && finite_d(a1p1R) && finite_d(a2p2R) &&
                           !(alpha1 > 0.0 && alpha1 <= tr) && !(alpha2 > 0.0 && alpha2 <= tr);
    if (admissible) {
        W[m->IE1] = a1p1R;
        W[m->IE2] = a2p2R;
        W[m->IA] = alpha1R;
        p2c(m, W, UR);
        return;
    }
    double AlphaR[2];
    const double Al[2] = {alpha1, alpha2}, Arr[2] = {a1r1, a2r2}, Ph[2] = {Phi1_In, Phi2_In}, Pi[2] = {Pi1_In, Pi2_In};
    const double Av[2] = {A1, A2}, Bv[2] = {B1, B2};
    const int path = relax_safeguarded2(AlphaR, Al, Arr, Ph, Pi, Av, Bv, tr);
    if (path != 1) AlphaR[0] = alpha1;
    AlphaR[1] = 1.0 - AlphaR[0];
    const double rho = a1r1 + a2r2;
    double rho_KE = 0.0;
    if (rho > 0.0) {
        double m2 = U[2] * U[2] + U[3] * U[3];
        if (D == 3) m2 = m2 + U[4] * U[4];
        rho_KE = 0.5 * m2 / rho;
    }
    const double KE = (rho > 0.0) ? rho_KE / rho : 0.0;
    const double E = U[m->IE1] + U[m->IE2];
    const double Phi1R = nasg_xi(AlphaR[0], a1r1, c->C1) * AlphaR[0];
    const double Phi2R = nasg_xi(AlphaR[1], a2r2, c->C2) * AlphaR[1];
    const double pR = (E - rho_KE - a1r1 * c->D1 - a2r2 * c->D2 - B1 * Phi1R - B2 * Phi2R) / (A1 * Phi1R + A2 * Phi2R);
    double E1R = A1 * Phi1R * pR + B1 * Phi1R + a1r1 * (c->D1 + KE);
    double E2R = A2 * Phi2R * pR + B2 * Phi2R + a2r2 * (c->D2 + KE);
    if (AlphaR[0] >= AlphaR[1]) E1R = E - E2R;
    else E2R = E - E1R;
    for (int n = 0; n < N; ++n) UR[n] = U[n];
    UR[m->IE1] = E1R;
    UR[m->IE2] = E2R;
    UR[m->IA] = AlphaR[0];
}

/* ---- arrays ------------------------------------------------------------------------------------------- */
typedef struct {
    int n[3], ng, gz;
    long long px, pxy, S;
} Geo;

static Geo geo_of(const cmp_case* c) {
    Geo g;
    g.n[0] = c->n[0];
    g.n[1] = c->n[1];
    g.n[2] = (c->dim == 3) ? c->n[2] : 1;
    g.ng = c->ng;
    g.gz = (c->dim == 3) ? c->ng : 0;
    g.px = g.n[0] + 2 * g.ng;
    g.pxy = g.px * (g.n[1] + 2 * g.ng);
    g.S = g.pxy * (g.n[2] + 2 * g.gz);
    return g;
}

static long long at(const Geo* g, int i, int j, int k) {
    return (long long)(k + g->gz) * g->pxy + (long long)(j + g->ng) * g->px + (i + g->ng);
}

static void load(const Model* m, const Geo* g, const double* U, int i, int j, int k, double* out) {
    const long long q = at(g, i, j, k);
    for (int n = 0; n < m->N; ++n) out[n] = U[n * g->S + q];
}

/* BCType of component n across a boundary normal to d (0 periodic, 1 extrap, 2 even, 3 odd) */
static int bc_kind(int code, int n, int d, int D, int m0) {
    const int mom = (n >= m0 && n < m0 + D);
    if (code == 0) return 0;
    if (code == 2) return 1;
    if (code == 3 || code == 4) return (mom && n - m0 == d) ? 3 : 2;
    return mom ? 3 : 2;
}

int cmp_nstate(const cmp_case* c) { return model_of(c).N; }

int cmp_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int cmp_fill_ghosts(const cmp_case* c, double* U) {
    const Model m = model_of(c);
    const Geo g = geo_of(c);
    const int lo[3] = {0, 0, 0};
    const int hi[3] = {g.n[0] - 1, g.n[1] - 1, g.n[2] - 1};
    for (int d = 0; d < m.D; ++d)
        for (int n = 0; n < m.N; ++n)
            for (int side = 0; side < 2; ++side) {
                const int code = side == 0 ? c->lo_bc[d] : c->hi_bc[d];
                if (code != 0 && code != 2 && code != 3 && code != 4 && code != 5) return -1;
                const int kind = bc_kind(code, n, d, m.D, m.IM);
                for (int k = -g.gz; k < g.n[2] + g.gz; ++k)
                    for (int j = -g.ng; j < g.n[1] + g.ng; ++j)
                        for (int i = -g.ng; i < g.n[0] + g.ng; ++i) {
                            int idx[3] = {i, j, k};
                            const int x = idx[d];
                            if (side == 0 ? !(x < lo[d]) : !(x > hi[d])) continue;
                            int src[3] = {i, j, k};
                            double s = 1.0;
                            const int len = hi[d] - lo[d] + 1;
                            if (kind == 0) src[d] = side == 0 ? x + len : x - len;
                            else if (kind == 1) src[d] = side == 0 ? lo[d] : hi[d];
                            else {
                                src[d] = side == 0 ? (2 * lo[d] - 1 - x) : (2 * hi[d] + 1 - x);
                                if (kind == 3) s = -1.0;
                            }
                            U[n * g.S + at(&g, i, j, k)] = s * U[n * g.S + at(&g, src[0], src[1], src[2])];
                        }
            }
    return 0;
}

/* ---- THINC ------------------------------------------------------------------------------------- */
static double signnz(double x) { return x > 0.0 ? 1.0 : -1.0; }

/* Test control (not part of the reference algorithm): when on, every THINC face value is moved up
 * by one ulp. Tests use it to measure how strongly a case amplifies a last-bit difference in
 * exp / log / tanh between two math libraries, which bounds what a correct implementation on
 * another library can be held to. */
static int g_thinc_ulp = 0;
void cmp_set_thinc_ulp(int on) { g_thinc_ulp = on; }

/* Reconstruction2Face_THINC_D: id_face 1 = high face of the cell, 0 = low face */
static double thinc_face_alpha(double beta, double sigma, double abar, int id_face) {
    const double a = (id_face == 1) ? 0.0 : 1.0;
    const double b = (id_face == 1) ? 1.0 : -1.0;
    const double arg_ln = (exp(2.0 * beta * abar) - 1.0) / (exp(2.0 * beta) - exp(2.0 * beta * abar));
    const double cc = 0.5 / beta * log(arg_ln);
    const double arg = beta * (a + 0.5 * b * (sigma + 1.0) + cc);
    const double af = 0.5 * (1.0 + tanh(arg));
    const double r = dmin(1.0, dmax(0.0, af));
    return g_thinc_ulp ? nextafter(r, 2.0) : r;
}

/* Reconstruction2Face_MUSCL_D with the minmod slope (ID_Limiter 1) */
static double muscl_minmod(double fm, double fc, double fp, double dx, int id_face) {
    const double sm = (fc - fm) / dx;
    const double sp = (fp - fc) / dx;
    const double slope = dmin(dmax(sm, 0.0), dmax(sp, 0.0)) + dmax(dmin(sm, 0.0), dmin(sp, 0.0));
    return fc + (double)id_face * 0.5 * slope * dx;
}

/* Interpolation2Edge_Linear_D */
static double edge4(double c, double a1, double a2, double a12) { return 0.25 * c + 0.25 * a1 + 0.25 * a2 + 0.25 * a12; }

/* Component d of FDM_Normal_{X,Y,Z}FaceFromCenter at face (i,j,k) of direction d, written out per
 * direction as the reference does (the argument order of the edge averages differs per direction). */
static double face_normal_d(const Model* m, const Geo* g, const double* U, int i, int j, int k, int d) {
    const double* A = U + (long long)m->IA * g->S;
#define F(ii, jj, kk) A[at(g, (ii), (jj), (kk))]
    const double* dx = m->c->dx;
    double n[3] = {0.0, 0.0, 0.0};
    const double fc = F(i, j, k);
    if (d == 0) {
        const double xm = F(i - 1, j, k);
        n[0] = (fc - xm) / dx[0];
        n[1] = (edge4(fc, xm, F(i, j + 1, k), F(i - 1, j + 1, k)) - edge4(fc, xm, F(i, j - 1, k), F(i - 1, j - 1, k))) / dx[1];
        if (m->D == 3)
            n[2] = (edge4(fc, xm, F(i, j, k + 1), F(i - 1, j, k + 1)) - edge4(fc, xm, F(i, j, k - 1), F(i - 1, j, k - 1))) / dx[2];
    } else if (d == 1) {
        const double ym = F(i, j - 1, k);
        n[0] = (edge4(fc, F(i + 1, j, k), ym, F(i + 1, j - 1, k)) - edge4(fc, F(i - 1, j, k), ym, F(i - 1, j - 1, k))) / dx[0];
        n[1] = (fc - ym) / dx[1];
        if (m->D == 3)
            n[2] = (edge4(fc, ym, F(i, j, k + 1), F(i, j - 1, k + 1)) - edge4(fc, ym, F(i, j, k - 1), F(i, j - 1, k - 1))) / dx[2];
    } else {
        const double zm = F(i, j, k - 1);
        n[0] = (edge4(fc, F(i + 1, j, k), zm, F(i + 1, j, k - 1)) - edge4(fc, F(i - 1, j, k), zm, F(i - 1, j, k - 1))) / dx[0];
        n[1] = (edge4(fc, F(i, j + 1, k), zm, F(i, j + 1, k - 1)) - edge4(fc, F(i, j - 1, k), zm, F(i, j - 1, k - 1))) / dx[1];
        n[2] = (fc - zm) / dx[2];
    }
#undef F
    double sum = 0.0;
    for (int t = 0; t < m->D; ++t) sum += n[t] * n[t];
    if (sum == 0.0) return 0.0;
    return n[d] / sqrt(sum);
}

static double xi_rho(double rho, double b) { return (b > 0.0) ? 1.0 - b * rho : 1.0; }

/* Reconstruct_State_From_VolumeFraction (5Eq :15-63, 6Eq :14-62) */
static void thinc_rebuild(const Model* m, const double* Uf, double af, double* Uo) {
    const cmp_case* c = m->c;
    double W[MAXN];
    c2p(m, Uf, W);
    const double al = W[m->IA];
    const double rho1 = W[0] / al;
    const double rho2 = W[1] / (1.0 - al);
    const double m1 = af * rho1;
    const double m2 = (1.0 - af) * rho2;
    const double rr = m1 + m2;
    const double K = 0.5 * ksum(W + 2, m->D);
    double p1, p2;
    if (!m->six) {
        p1 = W[m->IE];
        p2 = W[m->IE];
    } else {
        p1 = W[m->IE1] / al;
        p2 = W[m->IE2] / (1.0 - al);
    }
    double r1e1 = c->A1 * p1 + c->B1 + rho1 * c->D1;
    double r2e2 = c->A2 * p2 + c->B2 + rho2 * c->D2;
    if (c->C1 > 0.0) r1e1 = xi_rho(rho1, c->C1) * (c->A1 * p1 + c->B1) + rho1 * c->D1;
    if (c->C2 > 0.0) r2e2 = xi_rho(rho2, c->C2) * (c->A2 * p2 + c->B2) + rho2 * c->D2;
    Uo[0] = m1;
    Uo[1] = m2;
    for (int d = 0; d < m->D; ++d) Uo[2 + d] = W[2 + d] * rr;
    if (!m->six) {
        Uo[m->IE] = K * rr + r1e1 * af + r2e2 * (1.0 - af);
    } else {
        Uo[m->IE1] = K * m1 + r1e1 * af;
        Uo[m->IE2] = K * m2 + r2e2 * (1.0 - af);
    }
    Uo[m->IA] = af;
}

/* FVM_Reconstruction2Face_Conservative_THINC_K: C[0..3] are the cells i-2 .. i+1 of the face (i,j,k)
 * of direction d. Returns 0 when the face keeps the base scheme. */
static int thinc_states(const Model* m, const Geo* g, const double* U, int i, int j, int k, int d, double C[][MAXN],
                        double* UL, double* UR) {
    const cmp_case* c = m->c;
    const int N = m->N, IA = m->IA;
    const double nd = face_normal_d(m, g, U, i, j, k, d);
    const double amm = C[0][IA], am = C[1][IA], ac = C[2][IA], ap = C[3][IA];
    const int grad_l = (ac - am) * (am - amm) > 0.0;
    const int grad_r = (ap - ac) * (ac - am) > 0.0;
    const int sym = (amm == ap) && (am == ac) && (am != amm);
    const int gate = (!c->thinc_use_normal) || (fabs(nd) > c->thinc_normal_threshold);
    const double eps = c->thinc_eps;
    const int int_l = (am > eps && am < 1.0 - eps) && (grad_l || sym) && gate;
    const int int_r = (ac > eps && ac < 1.0 - eps) && (grad_r || sym) && gate;
    if (!(int_l || int_r)) return 0;
    double P[4][MAXN], WL[MAXN], WR[MAXN];
    for (int s = 0; s < 4; ++s) c2p(m, C[s], P[s]);
    const double dxd = c->dx[d];
    for (int n = 0; n < N; ++n) {
        WL[n] = muscl_minmod(P[0][n], P[1][n], P[2][n], dxd, 1);
        WR[n] = muscl_minmod(P[1][n], P[2][n], P[3][n], dxd, -1);
    }
    p2c(m, WL, UL);
    p2c(m, WR, UR);
    const double beta = c->thinc_use_normal ? (c->thinc_beta * fabs(nd) + 0.01) : c->thinc_beta;
    double Uf[MAXN];
    if (int_l) {
        memcpy(Uf, UL, sizeof(double) * N);
        thinc_rebuild(m, Uf, thinc_face_alpha(beta, signnz(ac - amm), am, 1), UL);
    }
    if (int_r) {
        memcpy(Uf, UR, sizeof(double) * N);
        thinc_rebuild(m, Uf, thinc_face_alpha(beta, signnz(ap - am), ac, 0), UR);
    }
    return 1;
}

/* face (i,j,k) of direction d lies between cells (i,j,k) - e_d and (i,j,k) */
static void face_flux(const Model* m, const Geo* g, const double* U, int i, int j, int k, int d, double* F,
                      double* fnc, double* cmax) {
    const int N = m->N;
    double C[6][MAXN], P[6][MAXN], WL[MAXN], WR[MAXN], UL[MAXN], UR[MAXN];
    for (int s = 0; s < 6; ++s) {
        int ii = i, jj = j, kk = k;
        if (d == 0) ii += s - 3; else if (d == 1) jj += s - 3; else kk += s - 3;
        load(m, g, U, ii, jj, kk, C[s]);
    }
    /* left state: stencil i-3..i+1 centred at i-1, right face; right state: i-2..i+2 centred at i, left face */
    if (m->c->thinc && thinc_states(m, g, U, i, j, k, d, C + 1, UL, UR)) {
        hllc(m, UL, UR, d, F, fnc, cmax);
        return;
    }
    const int bounded = (m->c->id_limiter == 6);
    const int n0 = bounded ? 2 : 0, n1 = bounded ? m->IA : N;
    for (int s = 0; s < 5; ++s) c2p(m, C[s], P[s]);
    if (bounded) weno5b_bounded(m, P, 1, WL);
    for (int n = n0; n < n1; ++n) WL[n] = weno5(P[0][n], P[1][n], P[2][n], P[3][n], P[4][n], 1);
    p2c(m, WL, UL);
    if (m->np) np_consistent(m, UL, C[2], m->c->dx[d], 1);
    for (int s = 1; s < 6; ++s) c2p(m, C[s], P[s]);
    if (bounded) weno5b_bounded(m, P + 1, -1, WR);
    for (int n = n0; n < n1; ++n) WR[n] = weno5(P[1][n], P[2][n], P[3][n], P[4][n], P[5][n], -1);
    p2c(m, WR, UR);
    if (m->np) np_consistent(m, UR, C[3], m->c->dx[d], -1);
    hllc(m, UL, UR, d, F, fnc, cmax);
}

int cmp_energy_bound_min(const cmp_case* c, const double* U, double* out) {
    (void)c; (void)U; (void)out;
    return -2; /* the bound-preserving path is restated in the reference-header oracle only */
}

int cmp_bound_restarts(void) { return 0; }

int cmp_compute_dudt(const cmp_case* c, const double* U, double* dUdt, double* cmax_out) {
    if (!c->id_weno || c->id_limiter < 5) return -2;  /* the port restates the WENO5 / WENO5B reconstructions only */
    if (c->id_bound) return -2;
    const Model m = model_of(c);
    const Geo g = geo_of(c);
    const int N = m.N, NC = m.NC, D = m.D;
    double* F[3] = {0, 0, 0};
    double* FN[3] = {0, 0, 0};
    long long fsz[3];
    int fe[3][3];
    double cm_all = 0.0;
    for (int d = 0; d < D; ++d) {
        fe[d][0] = g.n[0] + (d == 0);
        fe[d][1] = g.n[1] + (d == 1);
        fe[d][2] = g.n[2] + (d == 2);
        fsz[d] = (long long)fe[d][0] * fe[d][1] * fe[d][2];
        F[d] = (double*)malloc(sizeof(double) * fsz[d] * N);
        FN[d] = (double*)malloc(sizeof(double) * fsz[d] * NC);
        double cm = 0.0;
        const int ex = fe[d][0], ey = fe[d][1], ez = fe[d][2];
#ifdef _OPENMP
#pragma omp parallel for collapse(2) reduction(max : cm) schedule(static)
#endif
        for (int k = 0; k < ez; ++k)
            for (int j = 0; j < ey; ++j)
                for (int i = 0; i < ex; ++i) {
                    double f[MAXN], fn[3], cmax;
                    face_flux(&m, &g, U, i, j, k, d, f, fn, &cmax);
                    const long long q = (long long)i + (long long)ex * (j + (long long)ey * k);
                    for (int n = 0; n < N; ++n) F[d][n * fsz[d] + q] = f[n];
                    for (int n = 0; n < NC; ++n) FN[d][n * fsz[d] + q] = fn[n];
                    if (i < g.n[0] && j < g.n[1] && k < g.n[2]) cm = dmax(cmax, cm);
                }
        cm_all = dmax(cm_all, cm);
    }
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int k = 0; k < g.n[2]; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i) {
                double div[MAXN + 3], W[MAXN], Uc[MAXN];
                for (int n = 0; n < N + NC; ++n) {
                    double acc = 0.0;
                    for (int d = 0; d < D; ++d) {
                        const int ex = fe[d][0], ey = fe[d][1];
                        const long long lo = (long long)i + (long long)ex * (j + (long long)ey * k);
                        const long long hi = lo + (d == 0 ? 1 : (d == 1 ? ex : (long long)ex * ey));
                        const double* arr = (n < N) ? F[d] + n * fsz[d] : FN[d] + (n - N) * fsz[d];
                        const double t = (arr[hi] - arr[lo]) / c->dx[d];
                        acc = (d == 0) ? t : acc + t;
                    }
                    div[n] = acc;
                }
                const long long q = at(&g, i, j, k);
                for (int n = 0; n < N; ++n) dUdt[n * g.S + q] = -div[n];
                load(&m, &g, U, i, j, k, Uc);
                c2p(&m, Uc, W);
                if (m.np) {
                    /* alpha_k += phi_k (1 + K_k) div u* (FVM_SurfaceIntegralNC_Compressible5Eq_NPhase.H) */
                    double K[MAXP], rc2[MAXP];
                    for (int kk = 0; kk < m.np; ++kk) K[kk] = 0.0;
                    if (c->source_term == 1) {
                        np_rc2_phases(&m, W[m.IE], rc2);
                        const double rho_c2 = np_rho_c2(&m, W, rc2, 1);
                        for (int kk = 0; kk < m.np; ++kk) K[kk] = (rho_c2 / rc2[kk] - 1.0);
                    }
                    for (int kk = 0; kk < m.np; ++kk) {
                        const double al = Uc[m.IA + kk];
                        const double Phi = (c->source_term == 1) ? nasg_phi(al, Uc[kk], c->Ck[kk]) : al;
                        dUdt[(m.IA + kk) * g.S + q] += Phi * (1.0 + K[kk]) * div[N];
                    }
                } else if (!m.six) {
                    double K1 = 0.0;
                    double phi1 = Uc[m.IA];
                    if (c->source_term == 1) {
                        const double p = W[m.IE];
                        const double r1 = ((c->A1 + 1.0) * p + c->B1) / c->A1;
                        const double r2 = ((c->A2 + 1.0) * p + c->B2) / c->A2;
                        const double a1 = W[m.IA], a2 = 1.0 - a1;
                        const double rc2 = 1.0 / (nasg_phi(a1, W[0], c->C1) / r1 + nasg_phi(a2, W[1], c->C2) / r2);
                        K1 = rc2 / r1 - 1.0;
                        phi1 = nasg_phi(Uc[m.IA], Uc[0], c->C1);
                    }
                    dUdt[m.IA * g.S + q] += phi1 * (1.0 + K1) * div[N];
                } else {
                    const double a1r1 = W[0], a2r2 = W[1], rho = a1r1 + a2r2;
                    const double vg1 = div[N + 1] - W[m.IE1] * div[N];
                    const double vg2 = div[N + 2] - W[m.IE2] * div[N];
                    dUdt[m.IE1 * g.S + q] += (a2r2 / rho * vg1 - a1r1 / rho * vg2);
                    dUdt[m.IE2 * g.S + q] += -(a2r2 / rho * vg1 - a1r1 / rho * vg2);
                    dUdt[m.IA * g.S + q] += W[m.IA] * div[N];
                }
            }
    for (int d = 0; d < D; ++d) {
        free(F[d]);
        free(FN[d]);
    }
    if (cmax_out) *cmax_out = cm_all;
    return 0;
}

int cmp_relax(const cmp_case* c, double* U) {
    const Model m = model_of(c);
    if (!m.six || !c->relaxation) return 0;
    const Geo g = geo_of(c);
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
    for (int k = 0; k < g.n[2]; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i) {
                double v[MAXN], r[MAXN];
                const long long q = at(&g, i, j, k);
                for (int n = 0; n < m.N; ++n) v[n] = U[n * g.S + q];
                relax_cell(&m, v, r);
                for (int n = 0; n < m.N; ++n) U[n * g.S + q] = r[n];
            }
    return 0;
}

int cmp_rk3_step(const cmp_case* c, double* U, double dt, double* cmax_out) {
    if (!c->id_weno || c->id_limiter < 5 || c->id_bound) return -2;
    const Model m = model_of(c);
    const Geo g = geo_of(c);
    const long long tot = g.S * m.N;
    double* U0 = (double*)malloc(sizeof(double) * tot);
    double* Ub = (double*)malloc(sizeof(double) * tot);
    double* L = (double*)calloc((size_t)tot, sizeof(double));
    memcpy(U0, U, sizeof(double) * tot);
    double cm = 0.0, cs;
    for (int stage = 0; stage < 3; ++stage) {
        memcpy(Ub, stage == 0 ? U0 : U, sizeof(double) * tot);
        cmp_fill_ghosts(c, Ub);
        cmp_compute_dudt(c, Ub, L, &cs);
        cm = dmax(cm, cs);
        const double a = stage == 0 ? 1.0 : (stage == 1 ? 0.25 : 2.0 / 3.0);
        const double b = stage == 1 ? 0.75 : 1.0 / 3.0;
        const double s = stage == 0 ? dt : (stage == 1 ? 0.25 * dt : (2.0 / 3.0) * dt);
#ifdef _OPENMP
#pragma omp parallel for collapse(3) schedule(static)
#endif
        for (int n = 0; n < m.N; ++n)
            for (int k = 0; k < g.n[2]; ++k)
                for (int j = 0; j < g.n[1]; ++j)
                    for (int i = 0; i < g.n[0]; ++i) {
                        const long long q = n * g.S + at(&g, i, j, k);
                        if (stage == 0) {
                            U[q] = 1.0 * Ub[q] + s * L[q];
                        } else {
                            U[q] = a * Ub[q] + b * U0[q];
                            U[q] += s * L[q];
                        }
                    }
        cmp_relax(c, U);
    }
    free(U0);
    free(Ub);
    free(L);
    if (cmax_out) *cmax_out = cm;
    return 0;
}

int cmp_advance(const cmp_case* c, double* U, int nsteps, double stop_time, double* t, double* dts) {
    if (!c->id_weno || c->id_limiter < 5 || c->id_bound) return -2;
    const Model m = model_of(c);
    const Geo g = geo_of(c);
    double dt_prev = 1.e100, cmax = 0.0, time = *t;
    int taken = 0;
    for (int step = 0; step < nsteps && time < stop_time; ++step) {
        if (time == 0.0) {
            const long long tot = g.S * m.N;
            double* Ub = (double*)malloc(sizeof(double) * tot);
            double* L = (double*)calloc((size_t)tot, sizeof(double));
            memcpy(Ub, U, sizeof(double) * tot);
            cmp_fill_ghosts(c, Ub);
            cmp_compute_dudt(c, Ub, L, &cmax);
            free(Ub);
            free(L);
        }
        double dt_est = DBL_MAX;
        for (int d = 0; d < m.D; ++d) dt_est = dmin(dt_est, c->cfl * c->dx[d] / cmax);
        if (time == 0.0) dt_prev = dt_est;
        if (c->change_limiter && dt_prev > 0.0) dt_est = dmin(dt_est, 1.1 * dt_prev);
        double dt0 = dt_est;
        const double eps = 1.0e-3 * dt0;
        if (time + dt0 > stop_time - eps) dt0 = stop_time - time;
        dt_prev = dt0;
        cmp_rk3_step(c, U, dt0, &cmax);
        if (dts) dts[step] = dt0;
        time += dt0;
        ++taken;
    }
    *t = time;
    return taken;
}

/* The Phase-Field step is in the reference-header build (oracle/ref_driver.cpp) only. */
int cmp_pf_step(const cmp_case* c, const cmp_pf* pf, double* U, double dt, double* info) {
    (void)c; (void)pf; (void)U; (void)dt; (void)info;
    return -2;
}
int cmp_pf_grad_q(const cmp_case* c, const cmp_pf* pf, const double* U, double dt, double* gq0, double* gq1,
                  double* gq2, double* info) {
    (void)c; (void)pf; (void)U; (void)dt; (void)gq0; (void)gq1; (void)gq2; (void)info;
    return -2;
}
int cmp_pf_dudt(const cmp_case* c, const cmp_pf* pf, const double* U, const double* gq0, const double* gq1,
                const double* gq2, double* dUdt) {
    (void)c; (void)pf; (void)U; (void)gq0; (void)gq1; (void)gq2; (void)dUdt;
    return -2;
}

int cmp_advance_pf(const cmp_case* c, const cmp_pf* pf, double* U, int nsteps, double stop_time, double* t,
                   double* dts) {
    (void)c; (void)pf; (void)U; (void)nsteps; (void)stop_time; (void)t; (void)dts;
    return -2;
}
int cmp_amr_advance(const cmp_case* c, int nlev, const cmp_amr_box* boxes, int nbox, double** U, int nsteps,
                    double stop_time, double* t, double* dts) {
    (void)c; (void)nlev; (void)boxes; (void)nbox; (void)U; (void)nsteps; (void)stop_time; (void)t; (void)dts;
    return -2;
}

/* Refinement tags: the reference-header build compiles the reference's own Tagging.H; the port does
 * not restate them. */
int cmp_tag(const cmp_case* c, const double* cv, const double* U, const cmp_tag_crit* crit, int ncrit,
            unsigned char* tags) {
    (void)c; (void)cv; (void)U; (void)crit; (void)ncrit; (void)tags;
    return -2;
}

int cmp_derive(const cmp_case* c, const double* cv, const double* U, const int* vars, const int* derived, int nvars,
               double* out) {
    (void)c; (void)cv; (void)U; (void)vars; (void)derived; (void)nvars; (void)out;
    return -2;
}

int cmp_thinc_face(const double* beta, const double* sigma, const double* abar, const int* side, long long n,
                   double* out) {
    (void)beta; (void)sigma; (void)abar; (void)side; (void)n; (void)out;
    return -2;
}
