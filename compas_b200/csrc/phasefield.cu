// Phase-Field regularisation step of the five-equation model on the device (see phasefield.h).
//
// Reference (orchestration in source/Class_Compressible_PhaseField.cpp):
//   PhaseField_Evolve            :424-595   mobility 0.5 eta max|u|, eta = Eta_Multiplier x max dx
//   PhaseFieldMechanism_Evolve   :596-711   explicit pseudo-time steps of the mechanism over dt
//   PhaseField_Mechanism (CAC)   :1006-1152 Allen-Cahn with the advective chemical potential and the
//                                           conservative Lagrange multiplier -int(mech)/int(W)
//   PhaseField_Mechanism (flux)  :1155-1232, PhaseField_ACDI :1494-1645
//   PhaseField_Normal            :1957-2033
//   PhaseField_GradQPF           :2132-2310 (implicit: div(beta grad Q) = Div_Jhat, beta = W(phi~)+1e-3,
//                                           AMReX MLMG ABecLaplacian), :2314-2401 (explicit)
// and the device functions of include/Physics_PhaseField and include/Operators_PhaseField cited at
// each kernel. The elliptic solve is this engine's own: conjugate gradients preconditioned by one
// geometric multigrid V-cycle (red-black Gauss-Seidel, or weighted Jacobi where a periodic side has
// an odd cell count), stopped at the reference's criterion max|r| <= LinearSystem.tol_rel max|rhs|.
// All arithmetic is FP64; sums are reduced in a fixed order (block partials, then one block), so a
// step is deterministic.
#include "phasefield.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "physics.cuh"

namespace compas {

namespace {

constexpr int kThreads = 256;
constexpr int kRedBlocks = 592;  // 4 x 148 SMs: partial sums of the reductions
constexpr int kMaxLevels = 24;

struct PfDims {
    int n[3];
    int D;
    double dx[3];
    int periodic[3];
    long long nv;            // valid cells
    int px, py, pz, gz;      // padded scalar layout: one ghost layer (none in z in 2D)
    long long ps;            // padded cells per component
    long long nf[3];         // faces per direction
};

PfDims make_dims(int D, const int* n, const double* dx, const int* periodic) {
    PfDims m;
    m.D = D;
    for (int d = 0; d < 3; ++d) {
        m.n[d] = (d < D) ? n[d] : 1;
        m.dx[d] = (d < D) ? dx[d] : 1.0;
        m.periodic[d] = (d < D) ? periodic[d] : 0;
    }
    m.nv = (long long)m.n[0] * m.n[1] * m.n[2];
    m.gz = (D == 3) ? 1 : 0;
    m.px = m.n[0] + 2;
    m.py = m.n[1] + 2;
    m.pz = m.n[2] + 2 * m.gz;
    m.ps = (long long)m.px * m.py * m.pz;
    for (int d = 0; d < 3; ++d)
        m.nf[d] = (d < D) ? (long long)(m.n[0] + (d == 0)) * (m.n[1] + (d == 1)) * (m.n[2] + (d == 2)) : 0;
    return m;
}

__device__ __forceinline__ long long pidx(const PfDims& m, int i, int j, int k) {
    return (long long)(i + 1) + m.px * ((long long)(j + 1) + (long long)m.py * (k + m.gz));
}
__device__ __forceinline__ long long vidx(const PfDims& m, int i, int j, int k) {
    return (long long)i + m.n[0] * ((long long)j + (long long)m.n[1] * k);
}
__device__ __forceinline__ long long fidx(const PfDims& m, int d, int i, int j, int k) {
    const int fx = m.n[0] + (d == 0), fy = m.n[1] + (d == 1);
    return (long long)i + fx * ((long long)j + (long long)fy * k);
}
__device__ __forceinline__ void vcoord(const PfDims& m, long long q, int& i, int& j, int& k) {
    i = (int)(q % m.n[0]);
    const long long r = q / m.n[0];
    j = (int)(r % m.n[1]);
    k = (int)(r / m.n[1]);
}
__device__ __forceinline__ void fcoord(const PfDims& m, int d, long long q, int& i, int& j, int& k) {
    const int fx = m.n[0] + (d == 0), fy = m.n[1] + (d == 1);
    i = (int)(q % fx);
    const long long r = q / fx;
    j = (int)(r % fy);
    k = (int)(r / fy);
}

#define GRID_STRIDE(q, total) \
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (total); q += (long long)gridDim.x * blockDim.x)

unsigned blocks_for(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

// ---- Phase-Field device functions (include/Physics_PhaseField) --------------------------------------
// Mapping_Backward.H: psi = sqrt(2) eta atanh(2 phi - 1), phi clipped to [1e-12, 1 - 1e-12]
__device__ __forceinline__ double map_backward(double phi, double eta) {
    const double ep = 1.0e-12;
    double t = phi;
    if (t < ep) t = ep;
    else if (t > 1.0 - ep) t = 1.0 - ep;
    return sqrt(2.0) * eta * atanh(2.0 * t - 1.0);
}
// Mapping_Forward.H (ID_Derivative 0 and 1)
__device__ __forceinline__ double map_forward(double psi, double eta) {
    return 0.5 + 0.5 * tanh(psi / (sqrt(2.0) * eta));
}
__device__ __forceinline__ double map_forward_d1(double psi, double eta) {
    return 0.5 / (sqrt(2.0) * eta) / cosh(psi / (sqrt(2.0) * eta)) / cosh(psi / (sqrt(2.0) * eta));
}
// face value of the mapped phase field (PhaseField_GradQPF :2218-2241 / :2357-2381)
__device__ __forceinline__ double face_mapped(double pc, double pm, double eta, double eta_f) {
    const double psic = map_backward(pc, eta), psim = map_backward(pm, eta);
    const double fc = map_forward(psic, eta_f * eta), fm = map_forward(psim, eta_f * eta);
    return 0.5 * fm + 0.5 * fc;
}

// ---- small kernels ----------------------------------------------------------------------------------
// volume fraction (component ia of the padded state) into a padded scalar field
__global__ void k_extract(const double* U, long long S, long long upx, long long upxy, int ung, int ugz, int ia,
                          PfDims m, double* dst) {
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const long long uq = (long long)(k + ugz) * upxy + (long long)(j + ung) * upx + (i + ung);
        dst[pidx(m, i, j, k)] = U[(long long)ia * S + uq];
    }
}

// ghost layer of a padded scalar field: int_dir on periodic directions, foextrap otherwise
__global__ void k_fill(double* f, int ncomp, PfDims m) {
    GRID_STRIDE(q, m.ps * ncomp) {
        const int c = (int)(q / m.ps);
        const long long r = q % m.ps;
        int i = (int)(r % m.px) - 1;
        const long long r2 = r / m.px;
        int j = (int)(r2 % m.py) - 1;
        int k = (int)(r2 / m.py) - m.gz;
        const bool ghost = i < 0 || i >= m.n[0] || j < 0 || j >= m.n[1] || (m.D == 3 && (k < 0 || k >= m.n[2]));
        if (!ghost) continue;
        int x[3] = {i, j, k};
        for (int d = 0; d < m.D; ++d) {
            if (x[d] < 0) x[d] = m.periodic[d] ? x[d] + m.n[d] : 0;
            else if (x[d] >= m.n[d]) x[d] = m.periodic[d] ? x[d] - m.n[d] : m.n[d] - 1;
        }
        f[c * m.ps + r] = f[c * m.ps + pidx(m, x[0], x[1], x[2])];
    }
}

// FDM_Normal_CenterFromCenter_{K,D}: normalised centred gradient of f at the valid cells
__global__ void k_normal(const double* f, double* nrm, PfDims m) {
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const double fc = f[pidx(m, i, j, k)];
        double gr[3] = {0.0, 0.0, 0.0};
        double sum = 0.0;
        for (int d = 0; d < m.D; ++d) {
            const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
            const double fm = f[pidx(m, i - ei, j - ej, k - ek)], fp = f[pidx(m, i + ei, j + ej, k + ek)];
            const double gm = (fc - fm) / m.dx[d], gp = (fp - fc) / m.dx[d];
            gr[d] = 0.5 * gm + 0.5 * gp;
            sum += gr[d] * gr[d];
        }
        const long long pq = pidx(m, i, j, k);
        for (int d = 0; d < m.D; ++d) nrm[d * m.ps + pq] = (sum == 0.0) ? 0.0 : gr[d] / sqrt(sum);
    }
}

// fixed-order block reduction of two sums into partial[blockIdx] (2 per block)
__device__ __forceinline__ void block_sum2(double a, double b, double* partial) {
    __shared__ double sa[kThreads], sb[kThreads];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = sa[0];
        partial[2 * blockIdx.x + 1] = sb[0];
    }
}

__global__ void k_reduce2(const double* partial, int nb, double* out) {
    __shared__ double sa[kThreads], sb[kThreads];
    double a = 0.0, b = 0.0;
    for (int t = threadIdx.x; t < nb; t += kThreads) {
        a += partial[2 * t];
        b += partial[2 * t + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

// CAC-Adv mechanism and weight at the valid cells, with their sums
// (FDM_PhaseFieldMechanism_ACAdv_{K,D}, FDM_ChemicalPotential_Adv_D, ChemicalPotential_Adv,
//  PotentialFunction_DoubleWell (first derivative), PhaseFieldMechanism_AC, WeightFunction_Quadratic)
__global__ void k_cac_mech(const double* pf, const double* nrm, PfDims m, double mob, double lam, double eta,
                           double* mech, double* wgt, double* partial) {
    double sm = 0.0, sw = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m.nv; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const long long c = pidx(m, i, j, k);
        const double fc = pf[c];
        double lap = 0.0, divn = 0.0, ag = 0.0;
        for (int d = 0; d < m.D; ++d) {
            const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
            const long long cm = pidx(m, i - ei, j - ej, k - ek), cp = pidx(m, i + ei, j + ej, k + ek);
            const double fm = pf[cm], fp = pf[cp];
            const double h = m.dx[d];
            const double gfp = (fp - fc) / h, gfm = (fc - fm) / h;
            const double tl = (gfp - gfm) / h;
            lap = (d == 0) ? tl : lap + tl;
            const double nc = nrm[d * m.ps + c], nm = nrm[d * m.ps + cm], np = nrm[d * m.ps + cp];
            const double nfp = 0.5 * nc + 0.5 * np, nfm = 0.5 * nm + 0.5 * nc;
            const double tn = (nfp - nfm) / h;
            divn = (d == 0) ? tn : divn + tn;
            const double g = 0.5 * gfm + 0.5 * gfp;
            ag += g * g;
        }
        const double curv = -divn;
        ag = sqrt(ag);
        const double g1 = 2.0 * fc * (1.0 - fc) * (1.0 - 2.0 * fc);
        const double mu = lam * ((1.0 / eta / eta) * g1 - lap - ag * curv);
        const double me = -mob * mu;
        const double w = fc * (1.0 - fc);
        mech[q] = me;
        wgt[q] = w;
        sm += me;
        sw += w;
    }
    block_sum2(sm, sw, partial);
}

// PhaseFieldMechanism_CAC and the explicit pseudo-time update phi = phi_old + dt Div_J
__global__ void k_cac_update(const double* mech, const double* wgt, const double* tot, const double* pfo, double* pf,
                             PfDims m, double dtm) {
    const double im = tot[0], iw = tot[1];
    const double L = (iw == 0.0) ? 0.0 : -im / iw;
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const double dj = mech[q] + wgt[q] * L;
        pf[pidx(m, i, j, k)] = 1.0 * pfo[q] + dtm * dj;
    }
}

__global__ void k_copy_valid(const double* pf, double* dst, PfDims m) {
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        dst[q] = pf[pidx(m, i, j, k)];
    }
}

// level-set of ACDI (Mapping_Backward at the valid cells)
__global__ void k_ls(const double* pf, double* ls, PfDims m, double eta) {
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const long long c = pidx(m, i, j, k);
        ls[c] = map_backward(pf[c], eta);
    }
}

// ACDI face flux of direction d (FDM_PhaseFieldFlux_ACDI_{K,D}, PhaseFieldFlux_ACDI); with the
// explicit approach also Jhat += dt J (MultiFab::Saxpy)
__global__ void k_acdi_flux(const double* pf, const double* nrm, PfDims m, int d, double mob, double eta, double* J,
                            double* Jhat, double dtm) {
    GRID_STRIDE(q, m.nf[d]) {
        int i, j, k;
        fcoord(m, d, q, i, j, k);
        const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
        const long long c = pidx(m, i, j, k), cm = pidx(m, i - ei, j - ej, k - ek);
        const double pc = pf[c], pm = pf[cm];
        const double psic = map_backward(pc, eta), psim = map_backward(pm, eta);
        const double grad = (pc - pm) / m.dx[d];
        const double psi = 0.5 * psim + 0.5 * psic;
        const double nf = 0.5 * nrm[d * m.ps + cm] + 0.5 * nrm[d * m.ps + c];
        const double mobf = 0.5 * mob + 0.5 * mob;
        const double f1 = map_forward_d1(psi, eta);
        const double flux = mobf * (grad - f1 * nf);
        J[q] = flux;
        if (Jhat) Jhat[q] = Jhat[q] + dtm * flux;
    }
}

// FVM_Divergence_K of the face fluxes and the pseudo-time update
__global__ void k_div_update(const double* J0, const double* J1, const double* J2, const double* pfo, double* pf,
                             PfDims m, double dtm) {
    GRID_STRIDE(q, m.nv) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const double* J[3] = {J0, J1, J2};
        double dv = 0.0;
        for (int d = 0; d < m.D; ++d) {
            const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
            const double t = (J[d][fidx(m, d, i + ei, j + ej, k + ek)] - J[d][fidx(m, d, i, j, k)]) / m.dx[d];
            dv = (d == 0) ? t : dv + t;
        }
        pf[pidx(m, i, j, k)] = 1.0 * pfo[q] + dtm * dv;
    }
}

// Div_Jhat = (1/dt) phi_new + (-1/dt) phi (MultiFab::LinComb), and its sum
__global__ void k_djhat(const double* pfn, const double* pf0, PfDims m, double inv, double* rhs, double* partial) {
    double s = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m.nv; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const long long c = pidx(m, i, j, k);
        const double v = inv * pfn[c] + (-inv) * pf0[c];
        rhs[q] = v;
        s += v;
    }
    block_sum2(s, 0.0, partial);
}

// face coefficient beta = W(phi~_face) + 1e-3 of direction d
__global__ void k_beta(const double* pf0, PfDims m, int d, double eta, double eta_f, double* beta) {
    GRID_STRIDE(q, m.nf[d]) {
        int i, j, k;
        fcoord(m, d, q, i, j, k);
        const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
        const double face = face_mapped(pf0[pidx(m, i, j, k)], pf0[pidx(m, i - ei, j - ej, k - ek)], eta, eta_f);
        beta[q] = face * (1.0 - face) + 1.0e-3;
    }
}

// explicit approach: grad Q = J / (W(phi~_face) + eps), J = Jhat (1/dt) (PhaseFieldFlux2GradQPF)
__global__ void k_gq_explicit(const double* pf0, const double* Jhat, PfDims m, int d, double inv, double eta,
                              double eta_f, double* gq) {
    GRID_STRIDE(q, m.nf[d]) {
        int i, j, k;
        fcoord(m, d, q, i, j, k);
        const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
        const double face = face_mapped(pf0[pidx(m, i, j, k)], pf0[pidx(m, i - ei, j - ej, k - ek)], eta, eta_f);
        const double J = Jhat[q] * inv;
        const double eps = 1.0e-3;
        const double flux = (face < eps || face > 1.0 - eps) ? 0.0 : J;
        gq[q] = flux / (face * (1.0 - face) + eps);
    }
}

// face gradient of the solution (MLMG getGradSolution): (Q_c - Q_m)/dx, zero on Neumann sides
__global__ void k_gq_from_q(const double* Q, PfDims m, int d, double* gq) {
    GRID_STRIDE(q, m.nf[d]) {
        int x[3];
        fcoord(m, d, q, x[0], x[1], x[2]);
        int mm[3] = {x[0], x[1], x[2]};
        mm[d] -= 1;
        if (x[d] == 0 || x[d] == m.n[d]) {
            if (!m.periodic[d]) {
                gq[q] = 0.0;
                continue;
            }
            x[d] = (x[d] + m.n[d]) % m.n[d];
            mm[d] = (mm[d] + m.n[d]) % m.n[d];
        }
        gq[q] = (Q[vidx(m, x[0], x[1], x[2])] - Q[vidx(m, mm[0], mm[1], mm[2])]) / m.dx[d];
    }
}

// largest non-negative value of the block into *out (bits of a double; one atomic per block)
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long* out) {
    __shared__ double wm[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = dmax(m, wm[w]);
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// max |u| over the valid cells of the padded state (MaxVelocity, Conservative2Velocity)
__global__ void k_maxv(const double* U, long long S, long long upx, long long upxy, int ung, int ugz, PfDims m,
                       unsigned long long* out) {
    double v = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m.nv; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        vcoord(m, q, i, j, k);
        const long long uq = (long long)(k + ugz) * upxy + (long long)(j + ung) * upx + (i + ung);
        const double rho = U[uq] + U[S + uq];
        double s = 0.0;
        for (int d = 0; d < m.D; ++d) {
            const double u = U[(2 + d) * S + uq] / rho;
            s = (d == 0) ? u * u : s + u * u;
        }
        v = dmax(v, fabs(sqrt(s)));
    }
    block_max_atomic(v, out);
}

__global__ void k_maxabs(const double* a, long long n, unsigned long long* out) {
    double v = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        v = dmax(v, fabs(a[q]));
    block_max_atomic(v, out);
}

// ---- multigrid -----------------------------------------------------------------------------------------
// A x = -div(beta grad x) on the valid cells (no flux through Neumann sides, wrap on periodic ones).
struct MgLevel {
    PfDims m;
    double* beta[3] = {nullptr, nullptr, nullptr};
    double* x = nullptr;
    double* b = nullptr;
    double* r = nullptr;
    double* idiag = nullptr;  // 1 / diagonal of A (set once per solve)
    double ih2[3] = {1.0, 1.0, 1.0};
    bool rb = true;  // red-black colouring is a proper two-colouring (no odd periodic side)
};

// off-diagonal part sum_f beta_f x_nb / h^2 of row (i,j,k) (32-bit indices: cells < 2^31)
__device__ __forceinline__ double mg_off(const MgLevel& L, const double* x, int i, int j, int k) {
    const PfDims& m = L.m;
    const int c[3] = {i, j, k};
    const int n0 = m.n[0], n1 = m.n[1];
    double off = 0.0;
    for (int d = 0; d < m.D; ++d) {
        const int fx = n0 + (d == 0), fy = n1 + (d == 1);
        for (int s = 0; s < 2; ++s) {
            int nb[3] = {c[0], c[1], c[2]};
            nb[d] += s ? 1 : -1;
            if (nb[d] < 0 || nb[d] >= m.n[d]) {
                if (!m.periodic[d]) continue;
                nb[d] = (nb[d] < 0) ? nb[d] + m.n[d] : nb[d] - m.n[d];
            }
            int f[3] = {c[0], c[1], c[2]};
            if (s) f[d] += 1;
            const double bf = L.beta[d][f[0] + fx * (f[1] + fy * f[2])] * L.ih2[d];
            off += bf * x[nb[0] + n0 * (nb[1] + n1 * nb[2])];
        }
    }
    return off;
}

// the same with the dimension known at compile time (the per-level kernels below)
template <int D>
__device__ __forceinline__ double mg_off_t(const MgLevel& L, const double* __restrict__ x, int i, int j, int k) {
    const PfDims& m = L.m;
    const int n0 = m.n[0], n1 = m.n[1];
    const int c[3] = {i, j, k};
    double off = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const int fx = n0 + (d == 0), fy = n1 + (d == 1);
        const double* __restrict__ bt = L.beta[d];
        const double ih = L.ih2[d];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            int nb[3] = {c[0], c[1], c[2]};
            nb[d] += s ? 1 : -1;
            bool ok = true;
            if (nb[d] < 0 || nb[d] >= m.n[d]) {
                if (m.periodic[d]) nb[d] = (nb[d] < 0) ? nb[d] + m.n[d] : nb[d] - m.n[d];
                else ok = false;
            }
            if (ok) {
                int f[3] = {c[0], c[1], c[2]};
                if (s) f[d] += 1;
                off += (bt[f[0] + fx * (f[1] + fy * f[2])] * ih) * x[nb[0] + n0 * (nb[1] + n1 * nb[2])];
            }
        }
    }
    return off;
}

// grid-shaped launches: x blocks along i, one grid row per (j, k) - no index division
#define MG_CELL(m)                                              \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;         \
    const int j = blockIdx.y, k = blockIdx.z;                    \
    if (i >= (m).n[0]) return;                                   \
    const int q = i + (m).n[0] * (j + (m).n[1] * k);

template <int D>
__global__ void k_mg_rb_t(MgLevel L, int color) {
    MG_CELL(L.m)
    if (((i + j + k) & 1) != color) return;
    L.x[q] = (L.b[q] + mg_off_t<D>(L, L.x, i, j, k)) * L.idiag[q];
}
// the residual of level L and its restriction to level C in one launch over C's cells: each coarse
// cell averages the residuals b - A x of its 2^D children
template <int D>
__global__ void k_mg_resrestrict_t(MgLevel L, MgLevel C) {
    MG_CELL(C.m)
    const int n0 = L.m.n[0], n1 = L.m.n[1];
    double s = 0.0;
#pragma unroll
    for (int dk = 0; dk < (D == 3 ? 2 : 1); ++dk)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
            for (int di = 0; di < 2; ++di) {
                const int fi = 2 * i + di, fj = 2 * j + dj, fk = (D == 3) ? 2 * k + dk : 0;
                const int fq = fi + n0 * (fj + n1 * fk);
                s += L.b[fq] - (L.x[fq] / L.idiag[fq] - mg_off_t<D>(L, L.x, fi, fj, fk));
            }
    C.b[q] = s / (double)(D == 3 ? 8 : 4);
}
template <int D>
__global__ void k_mg_apply_t(MgLevel L, const double* __restrict__ x, double* __restrict__ y) {
    MG_CELL(L.m)
    y[q] = x[q] / L.idiag[q] - mg_off_t<D>(L, x, i, j, k);
}
template <int D>
__global__ void k_mg_jacobi_t(MgLevel L) {
    MG_CELL(L.m)
    L.r[q] = L.x[q] + 0.8 * ((L.b[q] + mg_off_t<D>(L, L.x, i, j, k)) * L.idiag[q] - L.x[q]);
}

constexpr int kRowThreads = 128;
dim3 mg_grid(const PfDims& m) { return dim3((unsigned)((m.n[0] + kRowThreads - 1) / kRowThreads), (unsigned)m.n[1], (unsigned)m.n[2]); }

// Two red-black Gauss-Seidel sweeps (four colour passes) of a 2D level in ONE launch, by temporal
// blocking: each CTA loads its kRbTX x kRbTY tile with a halo of kRbH = 4 cells (x into shared memory;
// b, 1/diag and the four face coefficients beta_f / h^2 of every cell into registers; periodic sides
// wrapped) and runs the passes there; pass p updates the cells of its colour within kRbH - 1 - p rings of
// the tile, so after the fourth pass the tile holds exactly what four global passes give (a
// colour's update reads only the other colour), and only the tile is written back. This replaces
// four launches and four passes over the level by one.
constexpr int kRbTX = 32, kRbTY = 16, kRbH = 4, kRbPasses = kRbH;
constexpr int kRbW = kRbTX + 2 * kRbH, kRbHt = kRbTY + 2 * kRbH, kRbCells = kRbW * kRbHt;
// two cells of the tile and its halo per thread (cells t and t + kRbThreads): every thread's loads are
// in flight at once (the load phase is latency-bound otherwise). A cell is always updated by the same
// thread, so its right-hand side, 1/diagonal, face coefficients and neighbour flags stay in that
// thread's registers; only x lives in shared memory (neighbours read it), which keeps the passes off
// the shared-memory instruction limit (one load per neighbour and one store per update)
constexpr int kRbCellsPerThread = 2;
constexpr int kRbThreads = kRbCells / kRbCellsPerThread;
static_assert(kRbThreads * kRbCellsPerThread == kRbCells, "whole cells per thread");
constexpr size_t kRbSmem = sizeof(double) * (size_t)kRbCells;

// xmode: 0 starts from L.x; 1 from zero (the first smoothing of a correction, in place of zeroing
// L.x); 2 from L.x plus the parent's value of the coarser level's x, xc (cn0 columns) - the
// piecewise-constant prolongation of k_mg_prolong applied as the cells are loaded.
// The smoothed tile goes to xout, not to L.x: a CTA reads a halo of its neighbours' tiles, which other
// CTAs (of an earlier wave, when the grid exceeds one) would otherwise have overwritten already.
__global__ void __launch_bounds__(kRbThreads, 2) k_mg_rb4_2d(MgLevel L, int first_color, int xmode,
                                                             const double* __restrict__ xc, int cn0,
                                                             double* __restrict__ xout) {
    extern __shared__ double sx[];
    const PfDims& m = L.m;
    const int n0 = m.n[0], n1 = m.n[1];
    const int i0 = blockIdx.x * kRbTX - kRbH, j0 = blockIdx.y * kRbTY - kRbH;
    const double ih0 = L.ih2[0], ih1 = L.ih2[1];
    // per owned cell: rhs, 1/diag, the coefficients of the -x, +x, -y, +y neighbours (beta_f / h^2),
    // flags (bit0 in domain, bits1-4 neighbour present, bit5 colour) and its update reach (rings
    // outside the tile)
    double rb[kRbCellsPerThread], rd[kRbCellsPerThread], rw[kRbCellsPerThread], re[kRbCellsPerThread];
    double rs[kRbCellsPerThread], rn[kRbCellsPerThread];
    unsigned fl[kRbCellsPerThread];
    int ring[kRbCellsPerThread];
#pragma unroll
    for (int u = 0; u < kRbCellsPerThread; ++u) {
        const int c = threadIdx.x + u * kRbThreads;
        const int lx = c % kRbW, ly = c / kRbW;
        int i = i0 + lx, j = j0 + ly;
        bool in = true;
        // periodic sides wrap (as often as the tile and its halo need); a cell beyond a
        // non-periodic side is left out
        if (i < 0 || i >= n0) {
            if (m.periodic[0]) i = ((i % n0) + n0) % n0;
            else in = false;
        }
        if (j < 0 || j >= n1) {
            if (m.periodic[1]) j = ((j % n1) + n1) % n1;
            else in = false;
        }
        unsigned f = 0;
        double xv = 0.0;
        rb[u] = rd[u] = rw[u] = re[u] = rs[u] = rn[u] = 0.0;
        if (in) {
            const int q = i + n0 * j;
            if (xmode != 1) {
                xv = L.x[q];
                if (xmode == 2) xv += xc[(i >> 1) + cn0 * (j >> 1)];
            }
            rb[u] = L.b[q];
            rd[u] = L.idiag[q];
            const int fx = n0 + 1;
            f = 1;
            if (i > 0 || m.periodic[0]) f |= 2;
            if (i < n0 - 1 || m.periodic[0]) f |= 4;
            if (j > 0 || m.periodic[1]) f |= 8;
            if (j < n1 - 1 || m.periodic[1]) f |= 16;
            if ((i + j) & 1) f |= 32;
            rw[u] = L.beta[0][i + fx * j] * ih0;
            re[u] = L.beta[0][(i + 1) + fx * j] * ih0;
            rs[u] = L.beta[1][i + n0 * j] * ih1;
            rn[u] = L.beta[1][i + n0 * (j + 1)] * ih1;
        }
        sx[c] = xv;
        fl[u] = f;
        const int ox = lx - kRbH, oy = ly - kRbH;
        const int rx = ox < 0 ? -ox : (ox >= kRbTX ? ox - kRbTX + 1 : 0);
        const int ry = oy < 0 ? -oy : (oy >= kRbTY ? oy - kRbTY + 1 : 0);
        ring[u] = rx > ry ? rx : ry;
    }
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < kRbPasses; ++p) {
        const unsigned color = (unsigned)(first_color ^ (p & 1));
        const int reach = kRbH - 1 - p;  // rings of the tile this pass updates
#pragma unroll
        for (int u = 0; u < kRbCellsPerThread; ++u) {
            const int c = threadIdx.x + u * kRbThreads;
            const unsigned f = fl[u];
            if (ring[u] > reach || !(f & 1) || ((f >> 5) & 1) != color) continue;
            // the neighbours in mg_off_t's order: -x, +x, -y, +y
            double off = 0.0;
            if (f & 2) off += rw[u] * sx[c - 1];
            if (f & 4) off += re[u] * sx[c + 1];
            if (f & 8) off += rs[u] * sx[c - kRbW];
            if (f & 16) off += rn[u] * sx[c + kRbW];
            sx[c] = (rb[u] + off) * rd[u];
        }
        __syncthreads();
    }
    for (int c = threadIdx.x; c < kRbTX * kRbTY; c += kRbThreads) {
        const int lx = c % kRbTX, ly = c / kRbTX;
        const int i = blockIdx.x * kRbTX + lx, j = blockIdx.y * kRbTY + ly;
        if (i < n0 && j < n1) xout[i + n0 * j] = sx[(lx + kRbH) + kRbW * (ly + kRbH)];
    }
}

__global__ void k_mg_idiag(MgLevel L) {
    const PfDims& m = L.m;
    GRID_STRIDE(q, m.nv) {
        int c[3];
        vcoord(m, q, c[0], c[1], c[2]);
        double diag = 0.0;
        for (int d = 0; d < m.D; ++d)
            for (int s = 0; s < 2; ++s) {
                const int nb = c[d] + (s ? 1 : -1);
                if ((nb < 0 || nb >= m.n[d]) && !m.periodic[d]) continue;
                int f[3] = {c[0], c[1], c[2]};
                if (s) f[d] += 1;
                diag += L.beta[d][fidx(m, d, f[0], f[1], f[2])] * L.ih2[d];
            }
        L.idiag[q] = 1.0 / diag;
    }
}

__global__ void k_copy(const double* a, double* b, long long n) {
    GRID_STRIDE(q, n) b[q] = a[q];
}
__global__ void k_zero(double* a, long long n) {
    GRID_STRIDE(q, n) a[q] = 0.0;
}

// fine x += coarse x of the parent (piecewise-constant prolongation)
__global__ void k_mg_prolong(const double* xc, PfDims c, double* xf, PfDims f) {
    GRID_STRIDE(q, f.nv) {
        int i, j, k;
        vcoord(f, q, i, j, k);
        xf[q] += xc[vidx(c, i / 2, j / 2, (f.D == 3 ? k / 2 : 0))];
    }
}

// coarse face coefficient = average of the fine faces it covers
__global__ void k_mg_beta(const double* bf, PfDims f, double* bc, PfDims c, int d) {
    GRID_STRIDE(q, c.nf[d]) {
        int x[3];
        fcoord(c, d, q, x[0], x[1], x[2]);
        double s = 0.0;
        int cnt = 0;
        const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;  // transverse directions
        const int r0 = (t0 < c.D) ? 2 : 1, r1 = (t1 < c.D && t1 != d) ? 2 : 1;
        for (int a = 0; a < r0; ++a)
            for (int b = 0; b < r1; ++b) {
                int y[3] = {2 * x[0], 2 * x[1], (c.D == 3) ? 2 * x[2] : 0};
                y[t0] += a;
                if (t1 < 3) y[t1] += b;
                s += bf[fidx(f, d, y[0], y[1], y[2])];
                ++cnt;
            }
        bc[q] = s / (double)cnt;
    }
}

__global__ void k_add_const(double* a, long long n, const double* tot, double scale) {
    const double c = -tot[0] * scale;
    GRID_STRIDE(q, n) a[q] += c;
}
// the coarsest level: all sweeps in one single-block launch (colours separated by block barriers)
__global__ void k_mg_coarse(MgLevel L, int sweeps) {
    const PfDims& m = L.m;
    const int n = (int)m.nv;
    for (int s = 0; s < sweeps; ++s) {
        if (L.rb) {
            for (int c = 0; c < 2; ++c) {
                const int color = (s & 1) ? 1 - c : c;
                for (int q = threadIdx.x; q < n; q += blockDim.x) {
                    const int i = q % m.n[0], r = q / m.n[0];
                    const int j = r % m.n[1], k = r / m.n[1];
                    if (((i + j + k) & 1) != color) continue;
                    L.x[q] = (L.b[q] + mg_off(L, L.x, i, j, k)) * L.idiag[q];
                }
                __syncthreads();
            }
        } else {
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                const int i = q % m.n[0], r = q / m.n[0];
                const int j = r % m.n[1], k = r / m.n[1];
                L.r[q] = L.x[q] + 0.8 * ((L.b[q] + mg_off(L, L.x, i, j, k)) * L.idiag[q] - L.x[q]);
            }
            __syncthreads();
            for (int q = threadIdx.x; q < n; q += blockDim.x) L.x[q] = L.r[q];
            __syncthreads();
        }
    }
}

// The coarse part of a V-cycle, levels l0 .. nl-1 (each of at most kBlockCells cells), in one
// single-block launch: the same smoothing, restriction and prolongation as the per-level kernels,
// with block barriers between the steps.
constexpr int kBlockCells = 4096;
constexpr int kBlockThreads = 1024;
constexpr size_t kBlockSmemMax = 200 * 1024;  // shared memory of the single-block cycle

// Who runs a step of the single-block cycle: the whole block (barriers between steps), or its first
// warp alone for the smallest levels (warp barriers: a block barrier per step costs more than the
// step's work there). Either way every cell gets the same updates in the same order.
struct BlockTeam {
    __device__ static int id() { return threadIdx.x; }
    __device__ static int size() { return blockDim.x; }
    __device__ static void sync() { __syncthreads(); }
};
struct WarpTeam {
    __device__ static int id() { return threadIdx.x & 31; }
    __device__ static int size() { return 32; }
    __device__ static void sync() { __syncwarp(); }
};
constexpr long long kWarpCells = 128;  // levels of at most this many cells run on one warp

// One red-black colour pass of a 2D level with an even number of columns: each thread takes cells of
// the colour only (the t-th cell of the colour in row-major order), and the neighbour sum is written
// out in mg_off's order (-x, +x, -y, +y) with its boundary rules, so the values are mg_off's.
template <class T>
__device__ void blk_rb_pass_2d(const MgLevel& L, int color) {
    const PfDims& m = L.m;
    const int n0 = m.n[0], n1 = m.n[1], hw = n0 / 2;
    const int ncol = hw * n1;
    const double ih0 = L.ih2[0], ih1 = L.ih2[1];
    const bool p0 = m.periodic[0], p1 = m.periodic[1];
    for (int t = T::id(); t < ncol; t += T::size()) {
        const int j = t / hw;
        const int i = 2 * (t - j * hw) + ((j + color) & 1);
        const int q = i + n0 * j;
        double off = 0.0;
        if (i > 0 || p0) off += (L.beta[0][i + (n0 + 1) * j] * ih0) * L.x[i > 0 ? q - 1 : q + n0 - 1];
        if (i < n0 - 1 || p0) off += (L.beta[0][(i + 1) + (n0 + 1) * j] * ih0) * L.x[i < n0 - 1 ? q + 1 : q - n0 + 1];
        if (j > 0 || p1) off += (L.beta[1][i + n0 * j] * ih1) * L.x[j > 0 ? q - n0 : q + n0 * (n1 - 1)];
        if (j < n1 - 1 || p1) off += (L.beta[1][i + n0 * (j + 1)] * ih1) * L.x[j < n1 - 1 ? q + n0 : q - n0 * (n1 - 1)];
        L.x[q] = (L.b[q] + off) * L.idiag[q];
    }
}

template <class T>
__device__ void blk_smooth(const MgLevel& L, int sweeps, bool reverse) {
    const PfDims& m = L.m;
    const int n = (int)m.nv;
    const bool fast2d = (m.D == 2 && L.rb && (m.n[0] % 2) == 0);
    for (int s = 0; s < sweeps; ++s) {
        if (fast2d) {
            for (int c = 0; c < 2; ++c) {
                blk_rb_pass_2d<T>(L, reverse ? 1 - c : c);
                T::sync();
            }
        } else if (L.rb) {
            for (int c = 0; c < 2; ++c) {
                const int color = reverse ? 1 - c : c;
                for (int q = T::id(); q < n; q += T::size()) {
                    const int i = q % m.n[0], r = q / m.n[0];
                    const int j = r % m.n[1], k = r / m.n[1];
                    if (((i + j + k) & 1) != color) continue;
                    L.x[q] = (L.b[q] + mg_off(L, L.x, i, j, k)) * L.idiag[q];
                }
                T::sync();
            }
        } else {
            for (int q = T::id(); q < n; q += T::size()) {
                const int i = q % m.n[0], r = q / m.n[0];
                const int j = r % m.n[1], k = r / m.n[1];
                L.r[q] = L.x[q] + 0.8 * ((L.b[q] + mg_off(L, L.x, i, j, k)) * L.idiag[q] - L.x[q]);
            }
            T::sync();
            for (int q = T::id(); q < n; q += T::size()) L.x[q] = L.r[q];
            T::sync();
        }
    }
}

// the downward step at level L: smooth, residual, restriction into C's right-hand side, C's x zeroed
template <class T>
__device__ void blk_down(const MgLevel& L, const MgLevel& C) {
    blk_smooth<T>(L, 2, false);
    const PfDims& m = L.m;
    for (int q = T::id(); q < (int)m.nv; q += T::size()) {
        const int i = q % m.n[0], r = q / m.n[0];
        const int j = r % m.n[1], k = r / m.n[1];
        L.r[q] = L.b[q] - (L.x[q] / L.idiag[q] - mg_off(L, L.x, i, j, k));
    }
    T::sync();
    const PfDims& c = C.m;
    for (int q = T::id(); q < (int)c.nv; q += T::size()) {
        const int I = q % c.n[0], r = q / c.n[0];
        const int J = r % c.n[1], K = r / c.n[1];
        double sacc = 0.0;
        const int kz = (c.D == 3) ? 2 : 1;
        for (int dk = 0; dk < kz; ++dk)
            for (int dj = 0; dj < 2; ++dj)
                for (int di = 0; di < 2; ++di)
                    sacc += L.r[(2 * I + di) + m.n[0] * ((2 * J + dj) + m.n[1] * (c.D == 3 ? 2 * K + dk : 0))];
        C.b[q] = sacc / (double)(c.D == 3 ? 8 : 4);
        C.x[q] = 0.0;
    }
    T::sync();
}

// the upward step at level L: C's correction prolonged (piecewise constant) onto L, then smoothed
template <class T>
__device__ void blk_up(const MgLevel& L, const MgLevel& C) {
    const PfDims& m = L.m;
    const PfDims& c = C.m;
    for (int q = T::id(); q < (int)m.nv; q += T::size()) {
        const int i = q % m.n[0], r = q / m.n[0];
        const int j = r % m.n[1], k = r / m.n[1];
        L.x[q] += C.x[(i / 2) + c.n[0] * ((j / 2) + c.n[1] * (m.D == 3 ? k / 2 : 0))];
    }
    T::sync();
    blk_smooth<T>(L, 2, true);
}

// the coarsest level: an even number of sweeps alternating the colour order (symmetric)
template <class T>
__device__ void blk_coarsest(const MgLevel& L) {
    for (int s = 0; s < 8; ++s) {
        blk_smooth<T>(L, 1, false);
        blk_smooth<T>(L, 1, true);
    }
}

// Shared memory of the single-block cycle over levels l0 .. nl-1: x, b, r, 1/diag and the face
// coefficients of every level.
__host__ __device__ inline long long block_cycle_doubles(const PfDims& m) {
    long long s = 4 * m.nv;
    for (int d = 0; d < m.D; ++d) s += m.nf[d];
    return s;
}

// The whole cycle runs in shared memory: every level's x, b, r, 1/diag and face coefficients (the
// last two copied in at the start, constant during a solve), level l0's x and b read at the start
// and its x written back at the end. Every step is the same arithmetic as the global-memory form,
// so the result is the same.
__global__ void __launch_bounds__(kBlockThreads) k_mg_vcycle_block(const MgLevel* levels, int l0, int nl) {
    extern __shared__ double bsm[];
    __shared__ MgLevel sl[kMaxLevels];
    if (threadIdx.x == 0) {
        long long off = 0;
        for (int l = l0; l < nl; ++l) {
            MgLevel L = levels[l];
            const long long n = L.m.nv;
            L.x = bsm + off;
            L.b = bsm + off + n;
            L.r = bsm + off + 2 * n;
            L.idiag = bsm + off + 3 * n;
            off += 4 * n;
            for (int d = 0; d < L.m.D; ++d) {
                L.beta[d] = bsm + off;
                off += L.m.nf[d];
            }
            sl[l] = L;
        }
    }
    __syncthreads();
    for (int l = l0; l < nl; ++l) {
        const MgLevel& G = levels[l];
        const MgLevel& L = sl[l];
        for (int q = threadIdx.x; q < (int)G.m.nv; q += blockDim.x) L.idiag[q] = G.idiag[q];
        for (int d = 0; d < G.m.D; ++d)
            for (int q = threadIdx.x; q < (int)G.m.nf[d]; q += blockDim.x) L.beta[d][q] = G.beta[d][q];
    }
    for (int q = threadIdx.x; q < (int)levels[l0].m.nv; q += blockDim.x) {
        sl[l0].x[q] = levels[l0].x[q];
        sl[l0].b[q] = levels[l0].b[q];
    }
    __syncthreads();
    // levels lw .. nl-1 (those of at most kWarpCells cells) run on the first warp alone; lw == nl when
    // even the coarsest level is larger
    int lw = nl;
    while (lw > l0 && sl[lw - 1].m.nv <= kWarpCells) --lw;
    const int lb = (lw < nl - 1) ? lw : nl - 1;  // the block's downward steps are l0 .. lb-1
    for (int l = l0; l < lb; ++l) blk_down<BlockTeam>(sl[l], sl[l + 1]);
    if (lw == nl) {
        blk_coarsest<BlockTeam>(sl[nl - 1]);
    } else if (threadIdx.x < 32) {
        for (int l = lw; l < nl - 1; ++l) blk_down<WarpTeam>(sl[l], sl[l + 1]);
        blk_coarsest<WarpTeam>(sl[nl - 1]);
        for (int l = nl - 2; l >= lw; --l) blk_up<WarpTeam>(sl[l], sl[l + 1]);
    }
    __syncthreads();
    for (int l = lb - 1; l >= l0; --l) blk_up<BlockTeam>(sl[l], sl[l + 1]);
    for (int q = threadIdx.x; q < (int)levels[l0].m.nv; q += blockDim.x) levels[l0].x[q] = sl[l0].x[q];
}

// conjugate-gradient scalars kept on the device: cg[0] rz, [1] pAp, [2] alpha, [3] rz_new, [4] beta,
// [5] the sum of the preconditioned vector (its mean is removed)
enum CgOp { kCgRz0 = 0, kCgPAp = 1, kCgZsum = 2, kCgRz = 3 };

// true in the block that finishes last (the others' partials are then visible); the counter is
// reset by that block for the next launch
__device__ __forceinline__ bool last_block(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    return last;
}

// the fixed-order sum of the first of each block's pair of partials (block_sum2), by the last block
__device__ __forceinline__ double sum_partials(const double* partial, int nb) {
    __shared__ double sa[kThreads];
    double a = 0.0;
    for (int t = threadIdx.x; t < nb; t += kThreads) a += __ldcg(partial + 2 * t);
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sa[threadIdx.x] += sa[threadIdx.x + s];
        __syncthreads();
    }
    return sa[0];
}

// the scalar update that follows a reduced sum: rz of the start, pAp with alpha = rz / pAp (and the
// residual maximum cleared for the update that follows), the sum of z, rz_new with beta = rz_new / rz
__device__ __forceinline__ void cg_finish(double* cg, int op, double tot, unsigned long long* rmax) {
    if (op == kCgRz0) {
        cg[0] = tot;
    } else if (op == kCgPAp) {
        cg[1] = tot;
        cg[2] = (cg[1] > 0.0) ? cg[0] / cg[1] : 0.0;
        *rmax = 0ull;
    } else if (op == kCgZsum) {
        cg[5] = tot;
    } else {
        cg[3] = tot;
        cg[4] = (cg[0] != 0.0) ? cg[3] / cg[0] : 0.0;
        cg[0] = cg[3];
    }
}

// A dot product (b == nullptr: the sum of a) and its scalar update in one launch of kRedBlocks
// blocks: grid-stride per-thread sums reduced per block (block_sum2), then the blocks' partials
// summed in a fixed order by the last block (a deterministic result)
__global__ void k_dot_cg(const double* a, const double* b, long long n, double* partial, unsigned int* counter,
                         double* cg, int op, unsigned long long* rmax) {
    double s = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        s += b ? a[q] * b[q] : a[q];
    block_sum2(s, 0.0, partial);
    if (!last_block(counter)) return;
    const double tot = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
        *counter = 0u;
        cg_finish(cg, op, tot, rmax);
    }
}

// z -= mean(z) (the sum in cg[5]) and the dot product r . z with its scalar update, in one launch of
// kRedBlocks blocks (the same bits as k_add_const, then k_dot_cg(r, z))
__global__ void k_center_dot_cg(double* z, const double* r, long long n, double scale, double* partial,
                                unsigned int* counter, double* cg, int op) {
    const double c = -cg[5] * scale;
    double s = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double zq = z[q] + c;
        z[q] = zq;
        s += r[q] * zq;
    }
    block_sum2(s, 0.0, partial);
    if (!last_block(counter)) return;
    const double tot = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
        *counter = 0u;
        cg_finish(cg, op, tot, nullptr);
    }
}

__global__ void k_axpy2(double* x, double* r, const double* p, const double* Ap, long long n, const double* alp,
                        unsigned long long* rmax) {
    const double al = *alp;
    double v = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        x[q] += al * p[q];
        r[q] -= al * Ap[q];
        v = dmax(v, fabs(r[q]));
    }
    block_max_atomic(v, rmax);
}
__global__ void k_xpby(const double* z, double* p, long long n, const double* bep) {
    const double be = *bep;
    GRID_STRIDE(q, n) p[q] = z[q] + be * p[q];
}
__global__ void k_sub(const double* a, const double* b, double* c, long long n) {
    GRID_STRIDE(q, n) c[q] = a[q] - b[q];
}
__global__ void k_neg(double* a, long long n) {
    GRID_STRIDE(q, n) a[q] = -a[q];
}

}  // namespace

struct PfLevel {
    PfDims m;
    int ia;                                  // component of alpha1 in the state
    long long S, upx, upxy;                  // padded state layout
    int ung, ugz;
    double* pfb0 = nullptr;                  // phase field at the step start (padded)
    double* pfb = nullptr;                   // mechanism iterate (padded)
    double* pfo = nullptr;                   // previous iterate (valid)
    double* nrm = nullptr;                   // normals (padded, D components)
    double* ls = nullptr;                    // ACDI level set (padded)
    double* mech = nullptr;
    double* wgt = nullptr;
    double* J[3] = {nullptr, nullptr, nullptr};
    double* Jhat[3] = {nullptr, nullptr, nullptr};
    double* gq[3] = {nullptr, nullptr, nullptr};
    double* partial = nullptr;               // 2 x kRedBlocks
    double* tot = nullptr;                   // 2 doubles
    unsigned long long* umax = nullptr;      // max reductions (bits)
    double* dt_slot = nullptr;
    // multigrid levels and the conjugate-gradient vectors of the finest one
    std::vector<MgLevel> mg;
    MgLevel* mg_dev = nullptr;               // the level descriptors on the device (block V-cycle)
    int mg_block0 = -1;                      // first level of the single-block coarse cycle
    size_t mg_block_smem = 0;                // its shared memory: x, b, r of every level it covers
    double *z = nullptr, *p = nullptr, *Ap = nullptr;
    double* rhs = nullptr;                   // right-hand side of the elliptic system
    unsigned int* cnt = nullptr;             // block counter of the one-launch reductions
    double* cg = nullptr;                    // device scalars of the conjugate gradients
    double* qsol = nullptr;                  // solution Q, kept as the next step's starting iterate
    cudaGraphExec_t cg_iter = nullptr;       // one captured iteration (fixed pointers)
    long long bytes = 0;
    std::vector<void*> allocs;
};

namespace {

cudaError_t dalloc(PfLevel* pf, double** ptr, long long n) {
    if (n < 1) n = 1;
    cudaError_t e = cudaMalloc((void**)ptr, sizeof(double) * n);
    if (e != cudaSuccess) return e;
    pf->allocs.push_back(*ptr);
    pf->bytes += sizeof(double) * n;
    return cudaMemset(*ptr, 0, sizeof(double) * n);
}

bool coarsenable(const PfDims& m) {
    for (int d = 0; d < m.D; ++d)
        if (m.n[d] % 2 != 0 || m.n[d] < 4) return false;
    return true;
}

#define PF_TRY(call)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            if (err) *err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return COMPAS_B200_ECUDA;                                                         \
        }                                                                                     \
    } while (0)

double read_max(unsigned long long* dev, cudaStream_t st) {
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, dev, sizeof(h), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    double v;
    std::memcpy(&v, &h, sizeof(v));
    return v;
}

// one V-cycle on level l (b_l given; x_l from zero when x_zero, else from its current value)
cudaError_t vcycle(PfLevel* pf, int l, cudaStream_t st, bool x_zero) {
    MgLevel& L = pf->mg[l];
    const unsigned nb = blocks_for(L.m.nv);
    const dim3 gg = mg_grid(L.m);
    const bool d3 = (L.m.D == 3);
    // 2D levels of at least 2 halo widths per side: two sweeps per temporally blocked launch
    const bool fused = !d3 && L.rb && L.m.n[0] >= 2 * kRbH && L.m.n[1] >= 2 * kRbH;
    // xmode as k_mg_rb4_2d's: 0 from x, 1 from zero, 2 from x plus the prolonged correction of C
    auto smooth = [&](int sweeps, bool reverse, int xmode, const MgLevel* C) {
        if (fused && sweeps == 2) {
            static bool attr = false;
            if (!attr) {
                cudaFuncSetAttribute(k_mg_rb4_2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRbSmem);
                attr = true;
            }
            const dim3 grid((unsigned)((L.m.n[0] + kRbTX - 1) / kRbTX), (unsigned)((L.m.n[1] + kRbTY - 1) / kRbTY));
            // out of place into the level's scratch vector r, which then becomes its x (the residual
            // of a fused 2D level is never stored, so r is free); a V-cycle swaps each level twice,
            // so every launch of a captured iteration sees the same pointers
            k_mg_rb4_2d<<<grid, kRbThreads, kRbSmem, st>>>(L, reverse ? 1 : 0, xmode, C ? C->x : nullptr,
                                                           C ? C->m.n[0] : 0, L.r);
            std::swap(L.x, L.r);
            return;
        }
        if (xmode == 1) k_zero<<<nb, kThreads, 0, st>>>(L.x, L.m.nv);
        else if (xmode == 2) k_mg_prolong<<<nb, kThreads, 0, st>>>(C->x, C->m, L.x, L.m);
        for (int s = 0; s < sweeps; ++s) {
            if (L.rb) {
                for (int c = 0; c < 2; ++c) {
                    const int color = reverse ? 1 - c : c;
                    if (d3) k_mg_rb_t<3><<<gg, kRowThreads, 0, st>>>(L, color);
                    else k_mg_rb_t<2><<<gg, kRowThreads, 0, st>>>(L, color);
                }
            } else {
                if (d3) k_mg_jacobi_t<3><<<gg, kRowThreads, 0, st>>>(L);
                else k_mg_jacobi_t<2><<<gg, kRowThreads, 0, st>>>(L);
                k_copy<<<nb, kThreads, 0, st>>>(L.r, L.x, L.m.nv);
            }
        }
    };
    if (l == pf->mg_block0) {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_mg_vcycle_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBlockSmemMax);
            attr = true;
        }
        if (x_zero) k_zero<<<nb, kThreads, 0, st>>>(L.x, L.m.nv);
        k_mg_vcycle_block<<<1, kBlockThreads, pf->mg_block_smem, st>>>(pf->mg_dev, l, (int)pf->mg.size());
        return cudaGetLastError();
    }
    if (l + 1 == (int)pf->mg.size()) {
        // an even number of sweeps alternating the colour order keeps the cycle symmetric
        if (x_zero) k_zero<<<nb, kThreads, 0, st>>>(L.x, L.m.nv);
        k_mg_coarse<<<1, kThreads, 0, st>>>(L, 16);
        return cudaGetLastError();
    }
    smooth(2, false, x_zero ? 1 : 0, nullptr);
    MgLevel& C = pf->mg[l + 1];
    if (d3) k_mg_resrestrict_t<3><<<mg_grid(C.m), kRowThreads, 0, st>>>(L, C);
    else k_mg_resrestrict_t<2><<<mg_grid(C.m), kRowThreads, 0, st>>>(L, C);
    cudaError_t e = vcycle(pf, l + 1, st, true);
    if (e != cudaSuccess) return e;
    smooth(2, true, 2, &C);
    return cudaGetLastError();
}

}  // namespace

int pf_create(const compas_b200_parm* p, const compas_b200_geom* g, PfLevel** out, std::string* err) {
    if ((long long)g->n[0] * g->n[1] * (p->dim == 3 ? g->n[2] : 1) >= (1LL << 31)) {
        if (err) *err = "the Phase-Field step supports boxes of fewer than 2^31 cells";
        return COMPAS_B200_EARG;
    }
    PfLevel* pf = new PfLevel();
    int per[3] = {0, 0, 0};
    for (int d = 0; d < p->dim; ++d) per[d] = (g->lo_bc[d] == 0);
    pf->m = make_dims(p->dim, g->n, g->dx, per);
    const PfDims& m = pf->m;
    pf->ia = (p->physics == COMPAS_B200_SIXEQS ? 4 : 3) + p->dim;  // alpha1, the last component
    pf->ung = g->ng;
    pf->ugz = (p->dim == 3) ? g->ng : 0;
    pf->upx = g->n[0] + 2LL * g->ng;
    pf->upxy = pf->upx * (g->n[1] + 2LL * g->ng);
    pf->S = pf->upxy * ((p->dim == 3 ? g->n[2] : 1) + 2LL * pf->ugz);
    auto fail_out = [&](cudaError_t e) {
        if (err) *err = std::string("Phase-Field work arrays: ") + cudaGetErrorString(e);
        pf_destroy(pf);
        return COMPAS_B200_ENOMEM;
    };
    cudaError_t e;
    if ((e = dalloc(pf, &pf->pfb0, m.ps)) || (e = dalloc(pf, &pf->pfb, m.ps)) || (e = dalloc(pf, &pf->pfo, m.nv)) ||
        (e = dalloc(pf, &pf->nrm, m.ps * m.D)) || (e = dalloc(pf, &pf->ls, m.ps)) || (e = dalloc(pf, &pf->mech, m.nv)) ||
        (e = dalloc(pf, &pf->wgt, m.nv)) || (e = dalloc(pf, &pf->partial, 2 * kRedBlocks)) ||
        (e = dalloc(pf, &pf->tot, 2)) || (e = dalloc(pf, &pf->dt_slot, 1)))
        return fail_out(e);
    if ((e = dalloc(pf, (double**)&pf->umax, 1))) return fail_out(e);
    for (int d = 0; d < m.D; ++d)
        if ((e = dalloc(pf, &pf->J[d], m.nf[d])) || (e = dalloc(pf, &pf->Jhat[d], m.nf[d])) ||
            (e = dalloc(pf, &pf->gq[d], m.nf[d])))
            return fail_out(e);
    // the conjugate-gradient vectors; z and the residual (mech) double as the finest level's x and b
    if ((e = dalloc(pf, &pf->z, m.nv)) || (e = dalloc(pf, &pf->p, m.nv)) || (e = dalloc(pf, &pf->Ap, m.nv)) ||
        (e = dalloc(pf, &pf->rhs, m.nv)) || (e = dalloc(pf, (double**)&pf->cnt, 1)) || (e = dalloc(pf, &pf->cg, 8)) ||
        (e = dalloc(pf, &pf->qsol, m.nv)))
        return fail_out(e);
    // multigrid hierarchy
    PfDims lm = m;
    for (int l = 0; l < kMaxLevels; ++l) {
        MgLevel L;
        L.m = lm;
        L.rb = true;
        for (int d = 0; d < lm.D; ++d)
            if (lm.periodic[d] && (lm.n[d] % 2)) L.rb = false;
        for (int d = 0; d < lm.D; ++d)
            if ((e = dalloc(pf, &L.beta[d], lm.nf[d]))) return fail_out(e);
        if (l == 0) {
            L.x = pf->z;
            L.b = pf->mech;
        } else if ((e = dalloc(pf, &L.x, lm.nv)) || (e = dalloc(pf, &L.b, lm.nv))) {
            return fail_out(e);
        }
        if ((e = dalloc(pf, &L.r, lm.nv)) || (e = dalloc(pf, &L.idiag, lm.nv))) return fail_out(e);
        for (int d = 0; d < lm.D; ++d) L.ih2[d] = 1.0 / (lm.dx[d] * lm.dx[d]);
        pf->mg.push_back(L);
        if (!coarsenable(lm) || lm.nv <= 16) break;
        int nc[3] = {lm.n[0] / 2, lm.n[1] / 2, lm.D == 3 ? lm.n[2] / 2 : 1};
        double dc[3] = {2 * lm.dx[0], 2 * lm.dx[1], lm.D == 3 ? 2 * lm.dx[2] : 1.0};
        lm = make_dims(lm.D, nc, dc, lm.periodic);
    }
    // the single-block cycle starts at the first level of at most kBlockCells cells whose levels fit
    // in shared memory together
    for (size_t l = 0; l < pf->mg.size() && pf->mg_block0 < 0; ++l) {
        if (pf->mg[l].m.nv > kBlockCells) continue;
        long long dbl = 0;
        for (size_t k = l; k < pf->mg.size(); ++k) dbl += block_cycle_doubles(pf->mg[k].m);
        if ((size_t)dbl * sizeof(double) <= kBlockSmemMax) {
            pf->mg_block0 = (int)l;
            pf->mg_block_smem = (size_t)dbl * sizeof(double);
        }
    }
    {
        const long long nbytes = (long long)(sizeof(MgLevel) * pf->mg.size() + 7) / 8;
        if ((e = dalloc(pf, (double**)&pf->mg_dev, nbytes))) return fail_out(e);
        if ((e = cudaMemcpy(pf->mg_dev, pf->mg.data(), sizeof(MgLevel) * pf->mg.size(), cudaMemcpyHostToDevice)))
            return fail_out(e);
    }
    *out = pf;
    return COMPAS_B200_OK;
}

void pf_destroy(PfLevel* pf) {
    if (!pf) return;
    if (pf->cg_iter) cudaGraphExecDestroy(pf->cg_iter);
    for (void* a : pf->allocs) cudaFree(a);
    delete pf;
}

const double* pf_gq(const PfLevel* pf, int d) { return pf->gq[d]; }
double* pf_dt_slot(PfLevel* pf) { return pf->dt_slot; }
long long pf_bytes(const PfLevel* pf) { return pf ? pf->bytes : 0; }

int pf_grad_q(PfLevel* pf, const compas_b200_parm* p, const double* U, double dt, cudaStream_t st, PfInfo* info,
              std::string* err) {
    const PfDims& m = pf->m;
    const unsigned nbv = blocks_for(m.nv), nbp = blocks_for(m.ps);
    // MaxVelocity and the parameters PhaseField_Evolve derives (:426-463)
    PF_TRY(cudaMemsetAsync(pf->umax, 0, sizeof(unsigned long long), st));
    k_maxv<<<nbv, kThreads, 0, st>>>(U, pf->S, pf->upx, pf->upxy, pf->ung, pf->ugz, m, pf->umax);
    PF_TRY(cudaGetLastError());
    const double vmax = read_max(pf->umax, st);
    const double lam = (p->pf_lambda <= 0.0) ? 1.0 : p->pf_lambda;
    double eta = p->pf_eta;
    if (eta <= 0.0) {
        double dxm = m.dx[0];
        for (int d = 1; d < m.D; ++d) dxm = std::max(dxm, m.dx[d]);
        eta = p->pf_eta_multiplier * dxm;
    }
    double mob = 1.0;
    mob *= 0.5 * eta * vmax;
    // PFBorder of the state
    k_extract<<<nbv, kThreads, 0, st>>>(U, pf->S, pf->upx, pf->upxy, pf->ung, pf->ugz, pf->ia, m, pf->pfb0);
    k_fill<<<nbp, kThreads, 0, st>>>(pf->pfb0, 1, m);
    PF_TRY(cudaMemcpyAsync(pf->pfb, pf->pfb0, sizeof(double) * m.ps, cudaMemcpyDeviceToDevice, st));
    const bool acdi = (p->pf_mechanism == 3);
    const bool explicit_rc = acdi && p->pf_explicit_rc;
    if (explicit_rc)
        for (int d = 0; d < m.D; ++d) PF_TRY(cudaMemsetAsync(pf->Jhat[d], 0, sizeof(double) * m.nf[d], st));
    // PhaseFieldMechanism_Evolve (:596-711)
    double mdt = 0.9 / (2.0 * mob * lam);
    {
        double s = 0.0;
        for (int d = 0; d < m.D; ++d) s = (d == 0) ? 1.0 / m.dx[d] / m.dx[d] : s + 1.0 / m.dx[d] / m.dx[d];
        mdt = mdt / (s + 1.0 / eta / eta);
    }
    double mt = 0.0;
    const double T = dt;
    int msteps = 0;
    while (mt < T) {
        if (mt + mdt > T) mdt = T - mt;
        k_copy_valid<<<nbv, kThreads, 0, st>>>(pf->pfb, pf->pfo, m);
        k_fill<<<nbp, kThreads, 0, st>>>(pf->pfb, 1, m);
        if (!acdi) {
            k_normal<<<nbv, kThreads, 0, st>>>(pf->pfb, pf->nrm, m);
            k_fill<<<nbp, kThreads, 0, st>>>(pf->nrm, m.D, m);
            k_cac_mech<<<kRedBlocks, kThreads, 0, st>>>(pf->pfb, pf->nrm, m, mob, lam, eta, pf->mech, pf->wgt, pf->partial);
            k_reduce2<<<1, kThreads, 0, st>>>(pf->partial, kRedBlocks, pf->tot);
            k_cac_update<<<nbv, kThreads, 0, st>>>(pf->mech, pf->wgt, pf->tot, pf->pfo, pf->pfb, m, mdt);
        } else {
            k_ls<<<nbv, kThreads, 0, st>>>(pf->pfb, pf->ls, m, eta);
            k_fill<<<nbp, kThreads, 0, st>>>(pf->ls, 1, m);
            k_normal<<<nbv, kThreads, 0, st>>>(pf->ls, pf->nrm, m);
            k_fill<<<nbp, kThreads, 0, st>>>(pf->nrm, m.D, m);
            for (int d = 0; d < m.D; ++d)
                k_acdi_flux<<<blocks_for(m.nf[d]), kThreads, 0, st>>>(pf->pfb, pf->nrm, m, d, mob, eta, pf->J[d],
                                                                      explicit_rc ? pf->Jhat[d] : nullptr, mdt);
            k_div_update<<<nbv, kThreads, 0, st>>>(pf->J[0], pf->J[1], pf->J[2], pf->pfo, pf->pfb, m, mdt);
        }
        PF_TRY(cudaGetLastError());
        mt += mdt;
        ++msteps;
    }
    int iters = 0;
    double res = 0.0;
    const double eta_f = p->pf_eta_factor;
    if (explicit_rc) {
        for (int d = 0; d < m.D; ++d)
            k_gq_explicit<<<blocks_for(m.nf[d]), kThreads, 0, st>>>(pf->pfb0, pf->Jhat[d], m, d, 1.0 / dt, eta, eta_f,
                                                                    pf->gq[d]);
        PF_TRY(cudaGetLastError());
    } else {
        // PhaseField_GradQPF, implicit (:2132-2310): div(beta grad Q) = Div_Jhat
        // The finest multigrid level reads its right-hand side from the residual r and writes its
        // solution into z (F.b == r, F.x == z), so the preconditioner z = V(r) needs no copies.
        MgLevel& F = pf->mg[0];
        double* rhs = pf->rhs;
        k_djhat<<<kRedBlocks, kThreads, 0, st>>>(pf->pfb, pf->pfb0, m, 1.0 / dt, rhs, pf->partial);
        k_reduce2<<<1, kThreads, 0, st>>>(pf->partial, kRedBlocks, pf->tot);
        k_add_const<<<nbv, kThreads, 0, st>>>(rhs, m.nv, pf->tot, 1.0 / (double)m.nv);  // solvable (zero mean)
        k_neg<<<nbv, kThreads, 0, st>>>(rhs, m.nv);  // A = -div(beta grad): A Q = -Div_Jhat
        for (int d = 0; d < m.D; ++d)
            k_beta<<<blocks_for(m.nf[d]), kThreads, 0, st>>>(pf->pfb0, m, d, eta, eta_f, F.beta[d]);
        for (size_t l = 1; l < pf->mg.size(); ++l)
            for (int d = 0; d < m.D; ++d)
                k_mg_beta<<<blocks_for(pf->mg[l].m.nf[d]), kThreads, 0, st>>>(pf->mg[l - 1].beta[d], pf->mg[l - 1].m,
                                                                               pf->mg[l].beta[d], pf->mg[l].m, d);
        for (size_t l = 0; l < pf->mg.size(); ++l)
            k_mg_idiag<<<blocks_for(pf->mg[l].m.nv), kThreads, 0, st>>>(pf->mg[l]);
        PF_TRY(cudaGetLastError());
        // preconditioned conjugate gradients on the mean-free space; the scalars stay on the device and
        // one iteration is a captured graph, so an iteration costs one host read (the residual norm)
        // The iterate starts from the previous step's solution (the problem changes little from one
        // step to the next); the stopping test is the reference's absolute one, max|r| <= tol max|rhs|,
        // so the warm start changes only the number of iterations.
        double* x = pf->qsol;
        double* r = pf->mech;     // residual (the mechanism's scratch is free here) == F.b
        double* z = pf->z;        // preconditioned residual == F.x
        if (m.D == 3) k_mg_apply_t<3><<<mg_grid(F.m), kRowThreads, 0, st>>>(F, x, pf->Ap);
        else k_mg_apply_t<2><<<mg_grid(F.m), kRowThreads, 0, st>>>(F, x, pf->Ap);
        k_sub<<<nbv, kThreads, 0, st>>>(rhs, pf->Ap, r, m.nv);
        PF_TRY(cudaMemsetAsync(pf->umax, 0, sizeof(unsigned long long), st));
        k_maxabs<<<nbv, kThreads, 0, st>>>(rhs, m.nv, pf->umax);
        const double bnorm = read_max(pf->umax, st);
        PF_TRY(cudaMemsetAsync(pf->umax, 0, sizeof(unsigned long long), st));
        k_maxabs<<<nbv, kThreads, 0, st>>>(r, m.nv, pf->umax);
        const double rnorm0 = read_max(pf->umax, st);
        // z = V(r) from a zero start, made mean-free, and r . z with the scalar update `op`
        auto precond_dot = [&](int op, cudaStream_t s2) -> cudaError_t {
            cudaError_t e = vcycle(pf, 0, s2, true);
            if (e != cudaSuccess) return e;
            k_dot_cg<<<kRedBlocks, kThreads, 0, s2>>>(z, nullptr, m.nv, pf->partial, pf->cnt, pf->cg, kCgZsum, nullptr);
            k_center_dot_cg<<<kRedBlocks, kThreads, 0, s2>>>(z, r, m.nv, 1.0 / (double)m.nv, pf->partial, pf->cnt,
                                                             pf->cg, op);
            return cudaGetLastError();
        };
        auto iteration = [&](cudaStream_t s2) -> cudaError_t {
            if (m.D == 3) k_mg_apply_t<3><<<mg_grid(F.m), kRowThreads, 0, s2>>>(F, pf->p, pf->Ap);
            else k_mg_apply_t<2><<<mg_grid(F.m), kRowThreads, 0, s2>>>(F, pf->p, pf->Ap);
            // pAp, alpha, and the residual maximum cleared for k_axpy2
            k_dot_cg<<<kRedBlocks, kThreads, 0, s2>>>(pf->p, pf->Ap, m.nv, pf->partial, pf->cnt, pf->cg, kCgPAp,
                                                      pf->umax);
            k_axpy2<<<nbv, kThreads, 0, s2>>>(x, r, pf->p, pf->Ap, m.nv, pf->cg + 2, pf->umax);
            cudaError_t e = precond_dot(kCgRz, s2);
            if (e != cudaSuccess) return e;
            k_xpby<<<nbv, kThreads, 0, s2>>>(z, pf->p, m.nv, pf->cg + 4);
            return cudaGetLastError();
        };
        const double tol = p->pf_tol_rel;
        if (bnorm > 0.0 && rnorm0 > tol * bnorm) {
            PF_TRY(precond_dot(kCgRz0, st));
            k_copy<<<nbv, kThreads, 0, st>>>(z, pf->p, m.nv);
            PF_TRY(cudaGetLastError());
            if (!pf->cg_iter) {
                cudaStream_t cap;
                PF_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
                cudaGraph_t graph;
                cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    cudaError_t e2 = iteration(cap);
                    e = cudaStreamEndCapture(cap, &graph);
                    if (e == cudaSuccess && e2 != cudaSuccess) e = e2;
                    if (e == cudaSuccess) {
                        e = cudaGraphInstantiate(&pf->cg_iter, graph, 0);
                        cudaGraphDestroy(graph);
                    }
                }
                cudaStreamDestroy(cap);
                PF_TRY(e);
            }
            res = 1.0;
            for (iters = 0; iters < 1000;) {
                PF_TRY(cudaGraphLaunch(pf->cg_iter, st));
                ++iters;
                res = read_max(pf->umax, st) / bnorm;
                if (!(res > tol)) break;
            }
        } else {
            res = (bnorm > 0.0) ? rnorm0 / bnorm : 0.0;
        }
        for (int d = 0; d < m.D; ++d) k_gq_from_q<<<blocks_for(m.nf[d]), kThreads, 0, st>>>(x, m, d, pf->gq[d]);
        PF_TRY(cudaGetLastError());
    }
    // max |grad Q| (PhaseField_ComputeDt)
    PF_TRY(cudaMemsetAsync(pf->umax, 0, sizeof(unsigned long long), st));
    for (int d = 0; d < m.D; ++d) k_maxabs<<<blocks_for(m.nf[d]), kThreads, 0, st>>>(pf->gq[d], m.nf[d], pf->umax);
    PF_TRY(cudaGetLastError());
    const double gmax = read_max(pf->umax, st);
    if (info) {
        info->max_v = vmax;
        info->mobility = mob;
        info->eta = eta;
        info->mech_steps = msteps;
        info->solve_iters = iters;
        info->solve_res = res;
        info->gmax = gmax;
    }
    return COMPAS_B200_OK;
}

}  // namespace compas
