// THINC interface reconstruction of the volume fraction (FiniteVolume.THINC = 1) for the fused stage
// kernel. A face whose left or right cell is an interface cell (volume fraction inside (EPS, 1-EPS),
// monotone or a two-cell plateau, face normal not too oblique) gets MUSCL-minmod states on both
// sides; the interface side(s) then take the THINC (tanh) face value of alpha1 and rebuild masses,
// momentum and energy from it. Every other face keeps the base scheme (WENO5 / WENO5B).
//
// Reference:
//   selection and states  include/Operators_Compressible5Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible5Eq.H:66-190,
//                         include/Operators_Compressible6Eq/FVM_Reconstruction2Face_Conservative_THINC_K_Compressible6Eq.H:64-188
//   tanh face value       include/Operators_FV/Reconstruction2Face_THINC_D.H:13-35
//   MUSCL-minmod          include/Operators_FV/Reconstruction2Face_MUSCL_D.H, Slope_TVD.H, Limiter_Minmod.H,
//                         Reconstruction2Face_Linear.H
//   face normal           include/Operators_FD/FDM_Normal_{X,Y,Z}FaceFromCenter_{K,D}.H,
//                         FDM_Gradient*_*FaceFromCenter_D.H, Interpolation2Edge_Linear_D.H
//
// The face normal needs alpha1 one cell across the transverse directions (edge cells of the tile),
// which the tile's shared-memory primitives do not hold; it is computed only for candidate faces,
// from the stage state in global memory (L2-resident), so the common face pays nothing for it.
#pragma once

namespace compas {

__device__ __forceinline__ double signnz(double x) { return (x > 0.0) ? 1.0 : -1.0; }

// tanh face value of alpha1 on the side id_face (1: the face at the cell's high end, 0: its low end).
__device__ __forceinline__ double thinc_alpha_face(double beta, double sigma, double abar, int id_face) {
    const double a = (id_face == 1) ? 0.0 : 1.0;
    const double b = (id_face == 1) ? 1.0 : -1.0;
    const double e2a = exp(2.0 * beta * abar);
    const double arg_ln = (e2a - 1.0) / (exp(2.0 * beta) - e2a);
    const double c = 0.5 / beta * log(arg_ln);
    const double t = beta * (a + 0.5 * b * (sigma + 1.0) + c);
    const double af = 0.5 * (1.0 + tanh(t));
    return dmin(1.0, dmax(0.0, af));
}

// Linear face value with the minmod slope; id_face +1 for the high face of the centre cell fc, -1 for
// the low face.
__device__ __forceinline__ double muscl_minmod(double fm, double fc, double fp, double dx, int id_face) {
    const double sm = (fc - fm) / dx;
    const double sp = (fp - fc) / dx;
    const double s = dmin(dmax(sm, 0.0), dmax(sp, 0.0)) + dmax(dmin(sm, 0.0), dmin(sp, 0.0));
    return fc + (double)id_face * 0.5 * s * dx;
}

// Edge average of four cell values, summed in the argument order of the reference.
__device__ __forceinline__ double edge4(double f0, double f1, double f2, double f3) {
    return 0.25 * f0 + 0.25 * f1 + 0.25 * f2 + 0.25 * f3;
}

// Component d of the unit normal of alpha1 at the face of direction d between cell c = (i,j,k) - e_d
// and c' = (i,j,k). A points to alpha1 of the padded box. The transverse gradients average the four
// cells around each edge of the face; the reference passes them in the order (c', c'-e_t ...) when
// the transverse direction t precedes d and (c', c ...) when it follows, which fixes the rounding.
template <int D>
__device__ __forceinline__ double thinc_normal_d(const double* A, const Grid& g, int d, int i, int j, int k) {
    const int ei = (d == 0), ej = (d == 1), ek = (d == 2);
    const double fc = A[g.at(i, j, k)];
    const double fm = A[g.at(i - ei, j - ej, k - ek)];
    const double dxd = (d == 0) ? g.dx[0] : (d == 1 ? g.dx[1] : g.dx[2]);
    const double gd = (fc - fm) / dxd;
    double sum = 0.0;
#pragma unroll
    for (int t = 0; t < D; ++t) {
        double gt;
        if (t == d) {
            gt = gd;
        } else {
            const int ti = (t == 0), tj = (t == 1), tk = (t == 2);
            const double cp = A[g.at(i + ti, j + tj, k + tk)];
            const double cm = A[g.at(i - ti, j - tj, k - tk)];
            const double mp = A[g.at(i - ei + ti, j - ej + tj, k - ek + tk)];
            const double mm = A[g.at(i - ei - ti, j - ej - tj, k - ek - tk)];
            double lo, hi;
            if (t < d) {
                lo = edge4(fc, cm, fm, mm);
                hi = edge4(fc, cp, fm, mp);
            } else {
                lo = edge4(fc, fm, cm, mm);
                hi = edge4(fc, fm, cp, mp);
            }
            const double dxt = (t == 0) ? g.dx[0] : (t == 1 ? g.dx[1] : g.dx[2]);
            gt = (hi - lo) / dxt;
        }
        sum += gt * gt;
    }
    if (sum == 0.0) return 0.0;
    return gd / sqrt(sum);
}

// THINC selection and face states of the face of direction d at cell index (i,j,k) (between
// (i,j,k) - e_d and (i,j,k)). P1..P4 give the primitives of the stencil cells i-2 .. i+1 along d
// (component n of cell s at P[s][n * stride[s]]). Returns false when the face keeps the base scheme;
// otherwise writes the conserved face states UL, UR.
template <class M, class PT>
__device__ __forceinline__ bool thinc_face_states(const Thinc& th, const double* Us, const Grid& g, const Eos& e,
                                                  const PT* sm, const int* off, const int* str, int d, int i, int j,
                                                  int k, double* UL, double* UR, unsigned int* err) {
    constexpr int N = M::N, IA = M::IA, D = M::D;
    const double amm = sm[off[0] + IA * str[0]], am = sm[off[1] + IA * str[1]];
    const double ac = sm[off[2] + IA * str[2]], ap = sm[off[3] + IA * str[3]];
    const bool grad_l = (ac - am) * (am - amm) > 0.0;
    const bool grad_r = (ap - ac) * (ac - am) > 0.0;
    const bool sym = (amm == ap) && (am == ac) && (am != amm);
    const double hi = 1.0 - th.eps;
    const bool cand_l = (am > th.eps && am < hi) && (grad_l || sym);
    const bool cand_r = (ac > th.eps && ac < hi) && (grad_r || sym);
    if (!(cand_l || cand_r)) return false;
    double beta = th.beta;
    if (th.use_normal) {
        const double nd = fabs(thinc_normal_d<D>(Us + (long long)IA * g.S, g, d, i, j, k));
        if (!(nd > th.thr)) return false;
        beta = th.beta * nd + 0.01;
    }
    const double dxd = (d == 0) ? g.dx[0] : (d == 1 ? g.dx[1] : g.dx[2]);
    double WL[N], WR[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const double p0 = sm[off[0] + n * str[0]], p1 = sm[off[1] + n * str[1]];
        const double p2 = sm[off[2] + n * str[2]], p3 = sm[off[3] + n * str[3]];
        WL[n] = muscl_minmod(p0, p1, p2, dxd, 1);
        WR[n] = muscl_minmod(p1, p2, p3, dxd, -1);
    }
    M::prim2cons(UL, WL, e, err);
    M::prim2cons(UR, WR, e, err);
    if (cand_l) {
        double Uf[N];
#pragma unroll
        for (int n = 0; n < N; ++n) Uf[n] = UL[n];
        M::thinc_rebuild(UL, Uf, thinc_alpha_face(beta, signnz(ac - amm), am, 1), e, err);
    }
    if (cand_r) {
        double Uf[N];
#pragma unroll
        for (int n = 0; n < N; ++n) Uf[n] = UR[n];
        M::thinc_rebuild(UR, Uf, thinc_alpha_face(beta, signnz(ap - am), ac, 0), e, err);
    }
    return true;
}

}  // namespace compas
