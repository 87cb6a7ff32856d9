// Refinement tagging on the device: ErrorEst of one level (source/COMPAS.cpp:767-932) for the
// two-phase models. For every valid cell and every criterion of the level, the tagged variable is a
// state component or one of the model's derived variables (compute_derived_var,
// include/Physics_Compressible5Eq/ComputeDerivedVar_Compressible5Eq.H and the six-equation
// counterpart, with the velocity-gradient invariants of include/DerivedVelocityGradient.H), and the
// tests are those of include/Tagging.H: state_grad (the largest one-sided difference to a neighbour
// along any direction >= threshold), state_value_less, state_value_greater, state_value_range. A
// cell is tagged when any criterion holds. Derived values are evaluated in the reference's order of
// operations, so tags equal the reference's on the same state.
#pragma once

namespace compas {

constexpr int kMaxTagCriteria = 16;
enum { kTagGrad = 0, kTagLess = 1, kTagGreater = 2, kTagRange = 3 };

struct TagCrit {
    int var, derived, kind;
    double v0, v1;
};

struct TagArgs {
    const double* U;
    Grid g;
    Eos e;
    double cv1, cv2;
    int ncrit;
    TagCrit c[kMaxTagCriteria];
    unsigned char* tags;  // valid cells, x fastest
};

// velocity (rho u_d)/rho with rho the sum of the partial densities (Conservative2Velocity)
template <class M>
__device__ __forceinline__ void tag_velocity(const double* base, const Grid& g, long long q, double v[3]) {
    const double rho = base[q] + base[g.S + q];
    v[0] = v[1] = v[2] = 0.0;
#pragma unroll
    for (int d = 0; d < M::D; ++d) v[d] = base[(2 + d) * g.S + q] / rho;
}

// VelocityGradientInvariants (include/DerivedVelocityGradient.H): second-order central differences of
// the velocity, vorticity magnitude, Q criterion, and lambda2 from the closed-form eigenvalues of
// S^2 + Omega^2 (Smith 1961)
template <class M>
__device__ void tag_velocity_invariants(const double* U, const Grid& g, int i, int j, int k, double& vort,
                                        double& qc, double& l2) {
    double G[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    const double h[3] = {g.dx[0], g.dx[1], M::D == 3 ? g.dx[2] : 1.0};
    for (int b = 0; b < M::D; ++b) {
        const int di = (b == 0), dj = (b == 1), dk = (b == 2);
        double vm[3], vp[3];
        tag_velocity<M>(U, g, g.at(i - di, j - dj, k - dk), vm);
        tag_velocity<M>(U, g, g.at(i + di, j + dj, k + dk), vp);
        for (int a = 0; a < M::D; ++a) G[a][b] = (vp[a] - vm[a]) / (2.0 * h[b]);
    }
    const double wx = G[2][1] - G[1][2];
    const double wy = G[0][2] - G[2][0];
    const double wz = G[1][0] - G[0][1];
    vort = sqrt(wx * wx + wy * wy + wz * wz);
    double S[3][3], W[3][3];
    qc = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            S[a][b] = 0.5 * (G[a][b] + G[b][a]);
            W[a][b] = 0.5 * (G[a][b] - G[b][a]);
            qc += 0.5 * (W[a][b] * W[a][b] - S[a][b] * S[a][b]);
        }
    double A[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            A[a][b] = 0.0;
            for (int c = 0; c < 3; ++c) A[a][b] += S[a][c] * S[c][b] + W[a][c] * W[c][b];
        }
    const double p1 = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    double e_max, e_min;
    const double q = (A[0][0] + A[1][1] + A[2][2]) / 3.0;
    if (p1 == 0.0) {
        e_max = dmax(dmax(A[0][0], A[1][1]), A[2][2]);
        e_min = dmin(dmin(A[0][0], A[1][1]), A[2][2]);
    } else {
        const double p2 = (A[0][0] - q) * (A[0][0] - q) + (A[1][1] - q) * (A[1][1] - q) + (A[2][2] - q) * (A[2][2] - q) +
                          2.0 * p1;
        const double p = sqrt(p2 / 6.0);
        double B[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) B[a][b] = (A[a][b] - (a == b ? q : 0.0)) / p;
        const double detB = B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) -
                            B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                            B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0]);
        const double r = dmin(dmax(0.5 * detB, -1.0), 1.0);
        const double phi = acos(r) / 3.0;
        const double two_pi_3 = 2.0 * 3.14159265358979323846 / 3.0;
        e_max = q + 2.0 * p * cos(phi);
        e_min = q + 2.0 * p * cos(phi + two_pi_3);
    }
    l2 = 3.0 * q - e_max - e_min;
}

// sum of u_d^2 over the directions in the reference's order (AMREX_D_TERM)
template <int D>
__device__ __forceinline__ double tag_k2(const double* u) {
    double s = u[0] * u[0];
    if (D > 1) s = s + u[1] * u[1];
    if (D > 2) s = s + u[2] * u[2];
    return s;
}

// Value of variable `var` at cell (i,j,k): state component (derived = 0) or derived variable
// (derived = 1, index into the model's list of derived names:
//   FIVEEQS a1rho1 a2rho2 rho_u rho_v rho_w rho_E a1 rho u v w P T c Mach vorticity_mag q_criterion lambda2
//   SIXEQS  a1rho1 a2rho2 rho_u rho_v rho_w a1rho1E1 a2rho2E2 a1 rho u v w P a1P1 a2P2 T c Mach
//           vorticity_mag q_criterion lambda2)
template <class M>
__device__ double tag_value(const TagArgs& A, int var, int derived, int i, int j, int k) {
    constexpr int N = M::N, D = M::D;
    const Grid& g = A.g;
    const long long q = g.at(i, j, k);
    if (!derived) return A.U[var * g.S + q];
    double U[N], W[N];
#pragma unroll
    for (int n = 0; n < N; ++n) U[n] = A.U[n * g.S + q];
    M::cons2prim(W, U, A.e, nullptr);
    double u[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < D; ++d) u[d] = W[2 + d];
    const Eos& e = A.e;
    constexpr bool SIX = (M::KIND == kModelSix);
    // shift of the derived indices after the phase energy / volume fraction entries
    constexpr int o = SIX ? 1 : 0;
    if (var == 0) return W[0];
    if (var == 1) return W[1];
    if (var == 2) return U[2];
    if (var == 3) return D > 1 ? U[3] : 0.0;
    if (var == 4) return D > 2 ? U[4] : 0.0;
    if (var == 5) return U[2 + D];
    if (var == 6) return U[3 + D];
    if (SIX && var == 7) return U[4 + D];
    if (var == 7 + o) return W[0] + W[1];
    if (var == 8 + o) return u[0];
    if (var == 9 + o) return u[1];
    if (var == 10 + o) return u[2];
    if (var == 11 + o) {
        if constexpr (SIX) return W[M::IE1] + W[M::IE2];
        else return W[M::IE];
    }
    if constexpr (SIX) {
        if (var == 13) return W[M::IE1];
        if (var == 14) return W[M::IE2];
    }
    const int rest = var - (SIX ? 15 : 12);  // T, c, Mach, vorticity_mag, q_criterion, lambda2
    // Conservative2Temperature: from the internal energy with the kinetic energy of u = rho_u / rho
    const double rho = U[0] + U[1];
    double uu[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < D; ++d) uu[d] = U[2 + d] / rho;
    const double k2 = tag_k2<D>(uu);
    if (rest == 0) {
        const double alpha1 = U[M::IA], alpha2 = 1.0 - alpha1;
        if constexpr (SIX) {
            const double e1 = U[M::IE1] - (0.5 * U[0]) * k2;
            const double e2 = U[M::IE2] - (0.5 * U[1]) * k2;
            const double BT1 = e.B1 / (1.0 + e.A1), BT2 = e.B2 / (1.0 + e.A2);
            const double Phi1 = nasg_xi(alpha1, U[0], e.C1, nullptr) * alpha1;
            const double Phi2 = nasg_xi(alpha2, U[1], e.C2, nullptr) * alpha2;
            const double T1 = ((e1 - U[0] * e.D1) - Phi1 * BT1) / A.cv1;
            const double T2 = ((e2 - U[1] * e.D2) - Phi2 * BT2) / A.cv2;
            return (T1 + T2) / rho;
        } else {
            const double rho_e = U[M::IE] - (0.5 * rho) * k2;
            const double Phi1 = nasg_phi(alpha1, U[0], e.C1, nullptr);
            const double Phi2 = nasg_phi(alpha2, U[1], e.C2, nullptr);
            const double rho_D = U[0] * e.D1 + U[1] * e.D2;
            const double rho_CT = U[0] * A.cv1 + U[1] * A.cv2;
            const double BT = Phi1 * (e.B1 / (1.0 + e.A1)) + Phi2 * (e.B2 / (1.0 + e.A2));
            return ((rho_e - rho_D) - BT) / rho_CT;
        }
    }
    double c;
    if constexpr (SIX) c = M::sound_speed(W, e, nullptr);
    else c = M::sound_speed(W, e, 0, nullptr);
    if (rest == 1) return c;
    if (rest == 2) return sqrt(tag_k2<D>(u)) / c;
    double vort, qc, l2;
    tag_velocity_invariants<M>(A.U, g, i, j, k, vort, qc, l2);
    if (rest == 3) return vort;
    if (rest == 4) return qc;
    if (rest == 5) return l2;
    return 0.0;
}

template <class M>
__global__ void tag_kernel(TagArgs A) {
    const Grid& g = A.g;
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.n[0]);
        const int j = (int)((t / g.n[0]) % g.n[1]);
        const int k = (int)(t / ((long long)g.n[0] * g.n[1]));
        bool tag = false;
        for (int v = 0; v < A.ncrit; ++v) {
            const TagCrit& c = A.c[v];
            const double s = tag_value<M>(A, c.var, c.derived, i, j, k);
            if (c.kind == kTagGrad) {
                // state_grad (include/Tagging.H): largest one-sided difference along each direction
                double ax = fabs(tag_value<M>(A, c.var, c.derived, i - 1, j, k) - s);
                double ay = fabs(tag_value<M>(A, c.var, c.derived, i, j - 1, k) - s);
                ax = dmax(ax, fabs(s - tag_value<M>(A, c.var, c.derived, i + 1, j, k)));
                ay = dmax(ay, fabs(s - tag_value<M>(A, c.var, c.derived, i, j + 1, k)));
                double az = 0.0;
                if (M::D == 3) {
                    az = fabs(tag_value<M>(A, c.var, c.derived, i, j, k - 1) - s);
                    az = dmax(az, fabs(s - tag_value<M>(A, c.var, c.derived, i, j, k + 1)));
                }
                if (dmax(dmax(ax, ay), az) >= c.v0) tag = true;
            } else if (c.kind == kTagLess) {
                if (s < c.v0) tag = true;
            } else if (c.kind == kTagGreater) {
                if (s > c.v0) tag = true;
            } else {
                if (s > c.v0 && s < c.v1) tag = true;
            }
        }
        A.tags[t] = tag ? 1 : 0;
    }
}

}  // namespace compas

namespace compas {

// Derived variables of the valid cells (the plot variables of the reference's PlotFileMF, computed
// by compute_derived_var): out[v * cells + t] for variable v and valid cell t (x fastest).
constexpr int kMaxDerive = 32;
struct DeriveArgs {
    TagArgs t;  // state, grid, EOS and heat capacities (no criteria)
    int nv;
    int var[kMaxDerive];
    int derived[kMaxDerive];
    double* out;
};

template <class M>
__global__ void derive_kernel(DeriveArgs A) {
    const Grid& g = A.t.g;
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.n[0]);
        const int j = (int)((t / g.n[0]) % g.n[1]);
        const int k = (int)(t / ((long long)g.n[0] * g.n[1]));
        for (int v = 0; v < A.nv; ++v) A.out[v * n + t] = tag_value<M>(A.t, A.var[v], A.derived[v], i, j, k);
    }
}

}  // namespace compas
