// Fused finite-volume right-hand side and TVD-RK3 stage of one level box on sm_100a.
//
// One CTA owns a tile of TX x TY x TZ cells. Per tile:
//   1. the conserved state of the tile cells is read once and converted to primitives into shared
//      memory (one Conservative2Primitive per cell instead of the reference's ~14 per face);
//   2. per direction d: the 3-cell halo slabs on both sides of the tile in d are converted into a
//      shared halo buffer; every face of the tile in d (T_d + 1 per line) is reconstructed (WENO5 in
//      primitive variables on both sides, then Primitive2Conservative), solved by HLLC, and its flux
//      and non-conservative face quantities are written to a shared face buffer; each cell then adds
//      (F_hi - F_lo)/dx_d to its register accumulator, in the order x, y, z of the reference's
//      divergence (include/Operators_FV/FVM_Divergence_D.H);
//   3. the epilogue forms dUdt = -div F + NC terms, the RK3 stage combination and, for the
//      six-equation model, the pressure relaxation, and writes the new state once.
// Face fluxes never leave shared memory; the face wave speeds are max-reduced per CTA (warp
// shuffles) into one atomic per CTA.
//
// The thread count NT is chosen so that the faces of one direction are an exact multiple of NT
// (8^3 tile: 9*8*8 = 576 = 2 x 288 threads; 16^2 tile: 17*16 = 272 threads), which keeps every
// face round full. Launch sites: source/Class_Compressible_PhaseField.cpp:3192-3250 (faces),
// :3310-3386 (divergence and NC terms), :3937-4107 (stage combinations),
// source/Class_Compressible6Eq_PhaseField.cpp:437-474 (relaxation).
#pragma once

#include "physics.cuh"
#include "physics_nphase.cuh"
#include "relax.cuh"
#include "physics_sixn.cuh"
#include "tma.cuh"

#include <type_traits>

namespace compas {

// Geometry of one state array (Array4 with ghosts; no z ghosts in 2D).
struct Grid {
    int n[3];
    int ng, gz;
    long long px, pxy, S;
    double dx[3];
    __device__ __forceinline__ long long at(int i, int j, int k) const {
        return (long long)(k + gz) * pxy + (long long)(j + ng) * px + (i + ng);
    }
    __device__ __forceinline__ bool padded(int i, int j, int k) const {
        return i >= -ng && i < n[0] + ng && j >= -ng && j < n[1] + ng && k >= -gz && k < n[2] + gz;
    }
};

enum StageMode { kModeStage = 0, kModeDudt = 1, kModeCmax = 2 };

struct StageArgs {
    const double* Us;   // stage state, ghosts filled
    const double* U0;   // state at the start of the step (stages 1, 2)
    double* Uout;       // new state (kModeStage) or dUdt (kModeDudt)
    Grid g;
    Eos e;
    int mode;
    int stage;
    const double* dt;          // device scalar
    const int* done;           // device flag: step is a no-op when set (may be null)
    unsigned long long* cmax;  // device double bits, atomicMax (non-negative)
    unsigned int* err;
    int id_k;
    int relax;
    double trace;
    Thinc thinc;               // used by the THINC kernels only
    const double* gq[3];       // Phase-Field kernels: face gradients of the potential Q per direction
    int pf_phasic;             // Phase-Field kernels, six-equation model: 1 phasic, 0 mixture formulation
    int pf_hll;                // Phase-Field kernels: 1 HLL phase fluxes, 0 upwind/downwind
    int muscl;                 // SCHEME 2: 0 Godunov, 1 minmod, 2 van Leer, 3 superbee, 4 MC, 10 WENO3, 11 WENO3B (-1 otherwise)
    int riemann;               // Physics.RiemannSolver: 0 LLF, 1 HLL, 2 HLLC
    int order;                 // tile traversal order (tile_coords): 0 x fastest, 1 bricks of tiles
    int tile_base;             // single-box kernels: first tile (order 0) and number of tiles of the launch
    int tile_count;            // (0: the whole box); a run of whole tile layers is a slab of the box
};

// Tile coordinates (in tiles) of the w-th CTA of a box of ntx x nty x ntz tiles. order 0: x fastest.
// order 1: bricks of BX x BY x BZ tiles (4^3 in 3D, 8^2 in 2D) walked x fastest, tiles inside a
// brick x fastest, so that the tiles resident at one time are close in every direction and their
// halo reads hit L2. The mapping is a bijection on [0, ntx*nty*ntz) (edge bricks are smaller).
__device__ __forceinline__ void tile_coords(int w, int ntx, int nty, int ntz, int order, int D, int& tx, int& ty,
                                            int& tz) {
    if (order == 0) {
        tx = w % ntx;
        ty = (w / ntx) % nty;
        tz = w / (ntx * nty);
        return;
    }
    const int BX = (D == 3) ? 4 : 8, BY = BX, BZ = (D == 3) ? 4 : 1;
    const int gz = w / (BZ * nty * ntx);
    int r = w - gz * BZ * nty * ntx;
    const int nz = min(BZ, ntz - gz * BZ);
    const int gy = r / (BY * nz * ntx);
    r -= gy * BY * nz * ntx;
    const int ny = min(BY, nty - gy * BY);
    const int gx = r / (BX * ny * nz);
    r -= gx * BX * ny * nz;
    const int nx = min(BX, ntx - gx * BX);
    tx = gx * BX + r % nx;
    ty = gy * BY + (r / nx) % ny;
    tz = gz * BZ + r / (nx * ny);
}

// Variants of the stage kernel (the VAR template argument of stage_tile). kVarTma: the plain
// right-hand side with the y and z halo slabs staged into shared memory by TMA (3D mixed form), each
// prefetched while the previous direction's faces are computed.
enum { kVarPlain = 0, kVarThinc = 1, kVarPhaseField = 2, kVarTma = 3 };

}  // namespace compas

#include "thinc.cuh"
#include "pf_flux.cuh"

namespace compas {

// Local Lax-Friedrichs (hll = 0) and HLL (hll = 1) face fluxes, Physics.RiemannSolver = LLF / HLL, with
// the face quantities of the non-conservative terms, for the three models:
//   include/Physics_Compressible5Eq/Riemann_LLF_Compressible5Eq.H, Riemann_HLL_Compressible5Eq.H,
//   include/Physics_Compressible6Eq/Riemann_LLF_Compressible6Eq.H, Riemann_HLL_Compressible6Eq.H,
//   include/Physics_Compressible5Eq_NPhase/Riemann_LLF_Compressible5Eq_NPhase.H, Riemann_HLL_...H.
// LLF: F = (FL + FR - lambda (UR - UL)) / 2, lambda = max(|VL| + cL, |VR| + cR), face velocity the mean;
// HLL: Sp = max(0, VL + cL, VR + cR), Sm = min(0, VL - cL, VR - cR), F = (Sp FL - Sm FR + Sp Sm (UR - UL))
// / (Sp - Sm), face velocity (Sp uL - Sm uR) / (Sp - Sm); six-equation: the face values of u alpha_k p_k
// likewise. cmax = max(cL + |uL|, cR + |uR|).
template <class M>
__device__ __forceinline__ void riemann_llf_hll(int hll, double* Fout, double* fnc, double& cmax, const double* UL,
                                                const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
    constexpr int N = M::N, D = M::D;
    constexpr int IU = M::IM;  // first velocity component of W
    double WL[N], WR[N];
    M::cons2prim(WL, UL, e, err);
    M::cons2prim(WR, UR, e, err);
    double FL[N], FR[N];
    M::flux(FL, UL, WL, d);
    M::flux(FR, UR, WR, d);
    double cL, cR;
    if constexpr (M::KIND == kModelSix || M::KIND == kModelSixN) {
        cL = M::sound_speed(WL, e, err);
        cR = M::sound_speed(WR, e, err);
    } else {
        cL = M::sound_speed(WL, e, id_k, err);
        cR = M::sound_speed(WR, e, id_k, err);
    }
    const double VL = pick<D>(WL + IU, d), VR = pick<D>(WR + IU, d);
    if (!hll) {
        const double lam = dmax(fabs(VL) + cL, fabs(VR) + cR);
#pragma unroll
        for (int i = 0; i < N; ++i) Fout[i] = (FL[i] + FR[i] - lam * (UR[i] - UL[i])) / 2.0;
        fnc[0] = (VL + VR) / 2.0;
        if constexpr (M::KIND == kModelSix) {
            fnc[1] = (VL * WL[M::IE1] + VR * WR[M::IE1]) / 2.0;
            fnc[2] = (VL * WL[M::IE2] + VR * WR[M::IE2]) / 2.0;
        }
    } else {
        double Sp = 0.0, Sm = 0.0;
        Sp = (Sp < VL + cL) ? VL + cL : Sp;
        Sp = (Sp < VR + cR) ? VR + cR : Sp;
        Sm = (VL - cL < Sm) ? VL - cL : Sm;
        Sm = (VR - cR < Sm) ? VR - cR : Sm;
#pragma unroll
        for (int i = 0; i < N; ++i) Fout[i] = (Sp * FL[i] - Sm * FR[i] + Sp * Sm * (UR[i] - UL[i])) / (Sp - Sm);
        fnc[0] = (Sp * VL - Sm * VR) / (Sp - Sm);
        if constexpr (M::KIND == kModelSix) {
            fnc[1] = (Sp * VL * WL[M::IE1] - Sm * VR * WR[M::IE1]) / (Sp - Sm);
            fnc[2] = (Sp * VL * WL[M::IE2] - Sm * VR * WR[M::IE2]) / (Sp - Sm);
        }
    }
    cmax = dmax(cL + sqrt(ksum<D>(WL + IU)), cR + sqrt(ksum<D>(WR + IU)));
}

// Mixed precision LLF / HLL of the two-phase models: wave speeds in FP32 from the FP32 face primitives
// (the sound speeds of the mixed HLLC), the fluxes assembled component by component in FP64 as
// a FL + b FR + c (UR - UL) (LLF: a = b = 1/2, c = -lambda/2; HLL: a = Sp/(Sp - Sm), b = -Sm/(Sp - Sm),
// c = Sp Sm/(Sp - Sm)), without per-side flux arrays.
template <class M>
__device__ __forceinline__ void llf_hll_mixed(int hll, double* Fout, double* fnc, float& cmax, const double* UL,
                                              const double* UR, const float* wL, const float* wR, const Eos& e, int d,
                                              int id_k) {
    constexpr int N = M::N, D = M::D;
    constexpr bool SIX = (M::KIND == kModelSix);
    float cL, cR;
    if constexpr (SIX) {
        cL = sixeq_c_f32<D>(wL, e);
        cR = sixeq_c_f32<D>(wR, e);
    } else {
        cL = fiveeq_c_f32<D>(wL, e, id_k);
        cR = fiveeq_c_f32<D>(wR, e, id_k);
    }
    const float VL = (d == 0) ? wL[2] : ((d == 1 || D == 2) ? wL[3] : wL[D == 3 ? 4 : 3]);
    const float VR = (d == 0) ? wR[2] : ((d == 1 || D == 2) ? wR[3] : wR[D == 3 ? 4 : 3]);
    double a, b, c;
    if (!hll) {
        const float lam = fmaxf(fabsf(VL) + cL, fabsf(VR) + cR);
        a = 0.5;
        b = 0.5;
        c = -0.5 * (double)lam;
    } else {
        const double Sp = fmaxf(0.0f, fmaxf(VL + cL, VR + cR)), Sm = fminf(0.0f, fminf(VL - cL, VR - cR));
        const double inv = 1.0 / (Sp - Sm);
        a = Sp * inv;
        b = -Sm * inv;
        c = (Sp * Sm) * inv;
    }
    const double VLd = VL, VRd = VR;
    double pl[2], pr[2];
    if constexpr (SIX) {
        pl[0] = wL[M::IE1]; pl[1] = wL[M::IE2];
        pr[0] = wR[M::IE1]; pr[1] = wR[M::IE2];
    } else {
        pl[0] = wL[M::IE]; pl[1] = 0.0;
        pr[0] = wR[M::IE]; pr[1] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double fl = UL[i] * VLd, fr = UR[i] * VRd;
        if (i >= 2 && i < 2 + D && i - 2 == d) {
            fl += pl[0] + pl[1];
            fr += pr[0] + pr[1];
        } else if (SIX && (i == M::IA - 2 || i == M::IA - 1)) {
            const int k = i - (M::IA - 2);  // phase energies: (alpha_k rho_k E_k + alpha_k p_k) V
            fl = (UL[i] + pl[k]) * VLd;
            fr = (UR[i] + pr[k]) * VRd;
        } else if (!SIX && i == M::IA - 1) {
            fl = (UL[i] + pl[0]) * VLd;
            fr = (UR[i] + pr[0]) * VRd;
        }
        Fout[i] = a * fl + b * fr + c * (UR[i] - UL[i]);
    }
    fnc[0] = a * VLd + b * VRd;
    if constexpr (SIX) {
        fnc[1] = a * (VLd * pl[0]) + b * (VRd * pr[0]);
        fnc[2] = a * (VLd * pl[1]) + b * (VRd * pr[1]);
    }
    float kL = wL[2] * wL[2] + wL[3] * wL[3], kR = wR[2] * wR[2] + wR[3] * wR[3];
    if (D == 3) { kL += wL[4] * wL[4]; kR += wR[4] * wR[4]; }
    cmax = fmaxf(cL + sqrtf(kL), cR + sqrtf(kR));
}

// Physics.RiemannSolver: 0 LLF, 1 HLL, 2 HLLC (source/Class_Compressible_PhaseField.cpp:92-111).
// WENO3B (three-cell code 11): the masses and volume fractions of the WENO3 face values Wf replaced by
// the bounded ones of bounded_phases<., 3>; g(s, n) is primitive n of stencil cell s = 0, 1, 2. The
// two-phase models bound alpha_2 = 1 - alpha_1 as the second phase
// (FVM_Reconstruction2Face_Conservative_WENO3B_D_Compressible5Eq.H:48-80).
template <class M, class PT, class G>
__device__ __forceinline__ void weno3b_faces(G g, int side, PT* Wf) {
    PT rf[M::NP], af[M::NP];
    if constexpr (M::KIND == kModelFiveN || M::KIND == kModelSixN) {
        bounded_phases<M::NP, 3, PT>([&](int k, int s) { return (PT)g(s, M::IR + k); },
                                     [&](int k, int s) { return (PT)g(s, M::IA + k); }, side, rf, af);
#pragma unroll
        for (int k = 0; k < M::NP; ++k) {
            Wf[M::IR + k] = rf[k];
            Wf[M::IA + k] = af[k];
        }
    } else {
        bounded_phases<2, 3, PT>(
            [&](int k, int s) { return (PT)g(s, k); },
            [&](int k, int s) {
                const PT a1 = (PT)g(s, M::IA);
                return (k == 0) ? a1 : (PT)1 - a1;
            },
            side, rf, af);
        Wf[0] = rf[0];
        Wf[1] = rf[1];
        Wf[M::IA] = af[0];
    }
}

// WENO5B: the components reconstructed with plain WENO5 ([lo, hi)); the masses and volume fractions
// outside that range are bounded.
template <class M>
__host__ __device__ constexpr int weno5b_plain_lo() {
    if constexpr (M::KIND == kModelSixN) return M::IP;
    else return M::IM;
}
template <class M>
__host__ __device__ constexpr int weno5b_plain_hi() {
    if constexpr (M::KIND == kModelSixN) return M::N;
    else return M::IA;
}

template <class M>
__device__ __forceinline__ void riemann(int id_riemann, double* Fout, double* fnc, double& cmax, const double* UL,
                                        const double* UR, const Eos& e, int d, int id_k, unsigned int* err) {
    if (id_riemann == 2) M::hllc(Fout, fnc, cmax, UL, UR, e, d, id_k, err);
    else if constexpr (M::KIND == kModelSixN) {
        // the N-phase six-equation LLF takes the face's cmax as its dissipation speed
        if (id_riemann == 0) M::llf(Fout, fnc, cmax, UL, UR, e, d, err);
        else riemann_llf_hll<M>(1, Fout, fnc, cmax, UL, UR, e, d, id_k, err);
    } else riemann_llf_hll<M>(id_riemann, Fout, fnc, cmax, UL, UR, e, d, id_k, err);
}

}  // namespace compas

namespace compas {

// PF: the Phase-Field kernel, whose face buffer holds the model's NCPF non-conservative face terms.
template <class M, int TX, int TY, int TZ, class PT = double, bool TMA = false, bool PF = false>
struct TileShape {
    static constexpr int D = M::D;
    static constexpr int CELLS = TX * TY * TZ;
    static constexpr int A0 = TY * TZ, A1 = TX * TZ, A2 = TX * TY;
    static constexpr int AMAX = (D == 3) ? (A0 > A1 ? (A0 > A2 ? A0 : A2) : (A1 > A2 ? A1 : A2)) : (A0 > A1 ? A0 : A1);
    // halo slab slot stride: padded by 8 cells in 3D so that the 4 slots a warp touches in one
    // face round fall in different shared-memory banks
    static constexpr int HS = (D == 3) ? AMAX + 8 : AMAX;
    static constexpr int HALO = 6 * HS;
    static constexpr int F0 = (TX + 1) * A0, F1 = (TY + 1) * A1, F2 = (TZ + 1) * A2;
    static constexpr int FMAX = (D == 3) ? (F0 > F1 ? (F0 > F2 ? F0 : F2) : (F1 > F2 ? F1 : F2)) : (F0 > F1 ? F0 : F1);
    static constexpr int NB = M::N + (PF ? M::NCPF : M::NC);
    static constexpr size_t FB = sizeof(double) * (size_t)NB * FMAX;  // face buffer (FP64)
    // Halo slab sets resident at once: D (every direction's slabs converted with the tile in step 1,
    // one barrier per direction fewer) where the primitives and the face buffer fit two CTAs per SM
    // (112 KB each), else 1 (the slabs of each direction converted before its faces, into one set).
    static constexpr size_t kTwoCtaBytes = 112 * 1024;
    static constexpr size_t pbytes(int nhs) { return sizeof(PT) * (size_t)M::N * (size_t)(CELLS + nhs * HALO); }
    static constexpr int NHS = (!TMA && (pbytes(D) + 15) / 16 * 16 + FB <= kTwoCtaBytes) ? D : 1;
    // primitives (type PT): component n of tile cell l at n * CSTR + l, of halo set h, slot s, slab
    // cell t at n * CSTR + CELLS + h * HALO + s * HS + t (one component stride for tile and halo, so
    // the stencil loads of a face differ only by compile-time offsets); then the face buffer
    static constexpr int CSTR = CELLS + NHS * HALO;
    static constexpr size_t PBYTES = pbytes(NHS);
    static constexpr size_t FOFF = (PBYTES + 15) / 16 * 16;
    static constexpr size_t FEND = FOFF + FB;
    // TMA staging of one direction's two halo slabs (raw FP64 boxes of kTmaBoxX x 3 x T x N), placed
    // at the next 128-byte boundary of the (runtime) shared-memory address, hence the 128-byte slack
    static constexpr size_t SLAB = sizeof(double) * (size_t)kTmaBoxX * 3 * TX * M::N;
    static constexpr size_t SMEM = TMA ? FEND + 128 + 2 * SLAB : FEND;
};

template <class M>
__device__ __forceinline__ void load_cons(double* U, const double* base, const Grid& g, long long q) {
#pragma unroll
    for (int n = 0; n < M::N; ++n) U[n] = base[n * g.S + q];
}

// SCHEME: 5 WENO5 on every primitive variable; 6 WENO5B (bounded masses and volume fractions,
// plain WENO5 on the velocity and the pressure(s)); 2 GODUNOV / MUSCL in primitive variables, the
// limiter a.muscl at run time.
// MIX: false - plain FP64, the reference's arithmetic to the bit; true - mixed precision: the cell
// primitives are recovered in FP64 (pressure from total energy) and kept in shared memory as FP32,
// the reconstruction runs in FP32, the Riemann solver, divergence, stage accumulation and
// relaxation in FP64.
// VAR: kVarPlain - the hyperbolic right-hand side; kVarThinc - with THINC interface reconstruction
// (FiniteVolume.THINC = 1); kVarPhaseField - the Phase-Field regularisation right-hand side (the
// same face states, the regularisation flux of the face gradient a.gq instead of the Riemann flux;
// FIVEEQS without non-conservative terms, SIXEQS with its phase-energy exchange).
// The work of one CTA on tile `tile` of the box described by `a` (tiles numbered x fastest).
template <class M, int SCHEME, bool MIX, int VAR, int TX, int TY, int TZ, int NT>
__device__ __forceinline__ void stage_tile(const StageArgs& a, int tile, double* smem_d, const TmaMaps* tm = nullptr) {
    static_assert(TX == TY && (M::D == 2 ? TZ == 1 : TZ == TX), "tiles are cubes (squares in 2D)");
    constexpr bool TH = (VAR == kVarThinc);
    constexpr bool PFX = (VAR == kVarPhaseField);
    constexpr bool TMA = (VAR == kVarTma);
    static_assert(!TMA || (M::D == 3 && MIX), "TMA halo staging: the 3D mixed form");
    static_assert(!PFX || M::KIND != kModelFiveN, "the Phase-Field kernel is the two-phase models'");
    static_assert(M::KIND != kModelFiveN || !TH, "FIVEEQS_NPHASE runs without THINC");
    static_assert(M::KIND != kModelSixN || VAR == kVarPlain,
                  "SIXEQS_IE_NPHASE: the plain hyperbolic right-hand side");
    static_assert(SCHEME != 2 || (VAR == kVarPlain && !TH), "GODUNOV / MUSCL: the plain right-hand side");
    constexpr bool NPH = (M::KIND == kModelFiveN);
    constexpr bool SXN = (M::KIND == kModelSixN);
    using PT = typename std::conditional<MIX, float, double>::type;
    using T = TileShape<M, TX, TY, TZ, PT, TMA, PFX>;
    constexpr int N = M::N, NC = PFX ? M::NCPF : M::NC, D = M::D, NB = T::NB;
    constexpr int CELLS = T::CELLS, HALO = T::HALO, FMAX = T::FMAX;
    constexpr int R = (CELLS + NT - 1) / NT;

    PT* smem = reinterpret_cast<PT*>(smem_d);
    PT* Pint = smem;             // tile cells: Pint[n * CSTR + l]
    PT* Phal = smem + CELLS;     // halo sets: Phal[n * CSTR + h * HALO + slot * HS + t]
    constexpr int CSTR = T::CSTR, NHS = T::NHS;
    double* Fb = reinterpret_cast<double*>(reinterpret_cast<char*>(smem_d) + T::FOFF);

    const Grid& g = a.g;
    const int ntx = (g.n[0] + TX - 1) / TX;
    const int nty = (g.n[1] + TY - 1) / TY;
    const int ntz = (g.n[2] + TZ - 1) / TZ;
    int tix, tiy, tiz;
    tile_coords(tile, ntx, nty, ntz, a.order, D, tix, tiy, tiz);
    const int i0 = tix * TX;
    const int j0 = tiy * TY;
    const int k0 = tiz * TZ;
    const int tid = threadIdx.x;
    unsigned int* err = a.err;
    __shared__ uint64_t tma_bar;
    double* stg = nullptr;  // TMA staging: low slab, then high slab
    if constexpr (TMA) {
        stg = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_d) + T::FEND + 127) & ~uintptr_t(127));
        if (tid == 0) mbar_init(&tma_bar, 1);  // visible to all after the barrier that ends step 1
    }

    // 1. tile cells and the x-direction halo slabs -> primitives, read as whole rows of TX + 6 cells
    // (coalesced), the tile cells into Pint and the halo cells into the x slabs of halo set 0; with
    // NHS = D also the y (and z) halo slabs, into halo sets 1 (and 2), in the same loop
    constexpr int RX = TX + 6;
    constexpr int ROWS = RX * TY * TZ;
    constexpr int A0 = T::A0;
    constexpr int ITEMS = ROWS + ((NHS == D) ? (D - 1) * 6 * A0 : 0);
    for (int l = tid; l < ITEMS; l += NT) {
        int lx, ly, lz, dst;
        if (l < ROWS) {
            lx = l % RX - 3;
            ly = (l / RX) % TY;
            lz = l / (RX * TY);
            if (lx >= 0 && lx < TX) {
                dst = lx + TX * (ly + TY * lz);
            } else {
                const int slot = (lx < 0) ? lx + 3 : lx - TX + 3;
                dst = CELLS + slot * T::HS + (ly + TX * lz);
            }
        } else {
            const int h = l - ROWS;
            const int dd = 1 + h / (6 * A0);
            const int hh = h - (dd - 1) * 6 * A0;
            const int slot = hh / A0, t = hh % A0;
            const int pos = (slot < 3) ? slot - 3 : TX + slot - 3;
            const int ta = t % TX, tb = t / TX;
            if (dd == 1) { lx = ta; ly = pos; lz = tb; }
            else { lx = ta; ly = tb; lz = pos; }
            dst = CELLS + dd * T::HALO + slot * T::HS + t;
        }
        const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
        double U[N];
        PT W[N];
        if (g.padded(i, j, k)) {
            load_cons<M>(U, a.Us, g, g.at(i, j, k));
            if constexpr (MIX) M::cons2prim_f32(W, U, a.e);
            else M::cons2prim(W, U, a.e, nullptr);
        } else {
#pragma unroll
            for (int n = 0; n < N; ++n) W[n] = 0;
        }
#pragma unroll
        for (int n = 0; n < N; ++n) smem[n * CSTR + dst] = W[n];
    }

    double acc[R][NB];
    double cmax_local = 0.0;

#pragma unroll 1
    for (int d = 0; d < D; ++d) {
        // cube (square) tiles: every direction has the same line length, slab area and transverse side
        constexpr int Td = TX;
        constexpr int Ad = T::A0;
        constexpr int Ta = TX;
        // 2a. halo slabs of direction d -> primitives (the x slabs came with the rows of step 1)
        if constexpr (TMA) {
            if (d > 0) {
                // the slabs were staged by TMA during the previous direction's faces (phase d - 1).
                // A wait that runs out sets the status bit and waits once more (bounded) for the copy
                // in flight; if that runs out too, the whole CTA leaves the tile without reading the
                // staging buffer or writing any output (a timed-out tile leaves its cells unwritten)
                bool lost = false;
                if (!mbar_wait_bounded(&tma_bar, (unsigned)(d - 1), 1 << 20)) {
                    flag_error(err, COMPAS_B200_ERR_TIMEOUT);
                    lost = !mbar_wait_bounded(&tma_bar, (unsigned)(d - 1), 1 << 20);
                }
                if (__syncthreads_or(lost)) return;
                const int offx = (i0 + g.ng) - ((i0 + g.ng - 1) & ~1);
                for (int h = tid; h < 6 * Ad; h += NT) {
                    const int slot = h / Ad, t = h % Ad;
                    const int pos = (slot < 3) ? slot - 3 : Td + slot - 3;
                    const int ta = t % Ta, tb = t / Ta;
                    const int b = (slot < 3) ? slot : slot - 3;
                    const double* sl = stg + ((slot < 3) ? 0 : T::SLAB / sizeof(double));
                    // box element (x, y, z) of component n: n*(10*3*8) + z*(10*Y) + y*10 + x
                    const int e0 = (d == 1) ? (ta + offx) + kTmaBoxX * b + kTmaBoxX * 3 * tb
                                            : (ta + offx) + kTmaBoxX * tb + kTmaBoxX * Ta * b;
                    int lx, ly, lz;
                    if (d == 1) { lx = ta; ly = pos; lz = tb; }
                    else { lx = ta; ly = tb; lz = pos; }
                    double U[N];
                    PT W[N];
                    if (g.padded(i0 + lx, j0 + ly, k0 + lz)) {
#pragma unroll
                        for (int n = 0; n < N; ++n) U[n] = sl[n * (kTmaBoxX * 3 * Ta) + e0];
                        M::cons2prim_f32(W, U, a.e);
                    } else {
#pragma unroll
                        for (int n = 0; n < N; ++n) W[n] = 0;
                    }
#pragma unroll
                    for (int n = 0; n < N; ++n) Phal[n * CSTR + slot * T::HS + t] = W[n];
                }
            }
        }
        // with one halo set, the slabs of d > 0 are converted here (d = 0 came with the rows of step 1)
        for (int h = (d == 0 || TMA || NHS == D) ? 6 * Ad : tid; h < 6 * Ad; h += NT) {
            const int slot = h / Ad, t = h % Ad;
            const int pos = (slot < 3) ? slot - 3 : Td + slot - 3;
            const int ta = t % Ta, tb = t / Ta;
            int lx, ly, lz;
            if (d == 0) { lx = pos; ly = ta; lz = tb; }
            else if (d == 1) { lx = ta; ly = pos; lz = tb; }
            else { lx = ta; ly = tb; lz = pos; }
            const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
            double U[N];
            PT W[N];
            if (g.padded(i, j, k)) {
                load_cons<M>(U, a.Us, g, g.at(i, j, k));
                if constexpr (MIX) M::cons2prim_f32(W, U, a.e);
                else M::cons2prim(W, U, a.e, nullptr);
            } else {
#pragma unroll
                for (int n = 0; n < N; ++n) W[n] = 0;
            }
#pragma unroll
            for (int n = 0; n < N; ++n) Phal[n * CSTR + slot * T::HS + t] = W[n];
        }
        // (also the barrier between the previous direction's divergence reads of the face buffer and
        // this direction's face writes)
        __syncthreads();

        // 2b. faces of direction d. Tiles are cubes (squares in 2D) of side TS, so every direction has
        // TS + 1 faces per line and the decode below divides by compile-time constants. For d = 0 the
        // face position runs fastest, for d > 0 the x index does, so that neighbouring threads read
        // neighbouring cells of the shared primitive arrays.
        constexpr int TS = TX;
        constexpr int EF = TS + 1;
        const int NF = EF * T::A0;
        const double dxd = (d == 0) ? g.dx[0] : (d == 1 ? g.dx[1] : g.dx[2]);
        if constexpr (TMA) {
            // stage the next direction's two halo slabs while this direction's faces are computed;
            // the staging was last read before the barrier above
            if (tid == 0 && d + 1 < D) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&tma_bar, (unsigned)(2 * T::SLAB));
                const int xs = (i0 + g.ng - 1) & ~1;  // even: an 8-byte element start on a 16-byte boundary
                double* hi = stg + T::SLAB / sizeof(double);
                if (d == 0) {
                    tma_load_4d(stg, &tm->y, &tma_bar, xs, j0 + g.ng - 3, k0 + g.gz, 0);
                    tma_load_4d(hi, &tm->y, &tma_bar, xs, j0 + g.ng + TY, k0 + g.gz, 0);
                } else {
                    tma_load_4d(stg, &tm->z, &tma_bar, xs, j0 + g.ng, k0 + g.gz - 3, 0);
                    tma_load_4d(hi, &tm->z, &tma_bar, xs, j0 + g.ng, k0 + g.gz + TZ, 0);
                }
            }
        }
        for (int f = tid; f < NF; f += NT) {
            int fd, ta, tb;
            if (d == 0) {
                fd = f % EF;
                const int t0 = f / EF;
                ta = t0 % TS;
                tb = t0 / TS;
            } else if (d == 1) {
                ta = f % TS;
                const int r0 = f / TS;
                fd = r0 % EF;
                tb = r0 / EF;
            } else {
                // z faces: x, then y, then the face position, so that a warp reads one z plane
                ta = f % TS;
                tb = (f / TS) % TS;
                fd = f / (TS * TS);
            }
            int fx, fy, fz;
            if (d == 0) { fx = fd; fy = ta; fz = tb; }
            else if (d == 1) { fx = ta; fy = fd; fz = tb; }
            else { fx = ta; fy = tb; fz = fd; }
            const int gi = i0 + fx, gj = j0 + fy, gk = k0 + fz;
            const bool valid = (d == 0 ? gi <= g.n[0] : gi < g.n[0]) && (d == 1 ? gj <= g.n[1] : gj < g.n[1]) &&
                               (D == 2 || (d == 2 ? gk <= g.n[2] : gk < g.n[2]));
            if (!valid) continue;
            const int t = ta + TS * tb;
            // shared-memory offset of the six stencil cells f-3 .. f+2 (component stride CSTR for all)
            const int hset = (NHS == 1) ? 0 : d;
            int off[6], str[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int pos = fd - 3 + s;
                if (pos >= 0 && pos < TS) {
                    int lx = fx, ly = fy, lz = fz;
                    if (d == 0) lx = pos; else if (d == 1) ly = pos; else lz = pos;
                    off[s] = lx + TX * (ly + TY * lz);
                } else {
                    const int slot = (pos < 0) ? pos + 3 : pos - TS + 3;
                    off[s] = CELLS + hset * HALO + slot * T::HS + t;
                }
                str[s] = CSTR;
            }
            double WfL[N], WfR[N], UL[N], UR[N];
            // first plainly reconstructed component and one past the last (WENO5B: all but the
            // bounded masses and volume fractions)
            constexpr int NB0 = (SCHEME == 6) ? weno5b_plain_lo<M>() : 0;
            constexpr int NB1 = (SCHEME == 6) ? weno5b_plain_hi<M>() : N;
            double F[N], fnc[NC], cm;
            bool thinc_face = false;
            if constexpr (TH)
                thinc_face = thinc_face_states<M, PT>(a.thinc, a.Us, g, a.e, smem, off + 1, str + 1, d, gi, gj, gk, UL,
                                                      UR, err);
            if constexpr (!MIX) {
                if (!thinc_face) {
                    if constexpr (SCHEME == 6 && (NPH || SXN)) {
                        double rf[M::NP], af[M::NP];
                        auto rl = [&](int k, int s) { return (double)smem[off[s] + (M::IR + k) * str[s]]; };
                        auto al_ = [&](int k, int s) { return (double)smem[off[s] + (M::IA + k) * str[s]]; };
                        bounded_phases<M::NP, 5, double>(rl, al_, 1, rf, af);
#pragma unroll
                        for (int k = 0; k < M::NP; ++k) { WfL[M::IR + k] = rf[k]; WfL[M::IA + k] = af[k]; }
                        auto rr = [&](int k, int s) { return (double)smem[off[s + 1] + (M::IR + k) * str[s + 1]]; };
                        auto ar_ = [&](int k, int s) { return (double)smem[off[s + 1] + (M::IA + k) * str[s + 1]]; };
                        bounded_phases<M::NP, 5, double>(rr, ar_, -1, rf, af);
#pragma unroll
                        for (int k = 0; k < M::NP; ++k) { WfR[M::IR + k] = rf[k]; WfR[M::IA + k] = af[k]; }
                    } else if constexpr (SCHEME == 6) {
                        double r1[6], r2[6], al[6];
#pragma unroll
                        for (int s = 0; s < 6; ++s) {
                            r1[s] = smem[off[s]];
                            r2[s] = smem[off[s] + str[s]];
                            al[s] = smem[off[s] + M::IA * str[s]];
                        }
                        weno5b_masses(r1, r2, al, 1, WfL[0], WfL[1], WfL[M::IA]);
                        weno5b_masses(r1 + 1, r2 + 1, al + 1, -1, WfR[0], WfR[1], WfR[M::IA]);
                    }
                    if constexpr (SCHEME == 2) {
                        const int lim = a.muscl;
#pragma unroll
                        for (int n = 0; n < N; ++n) {
                            const double w1 = smem[off[1] + n * str[1]], w2 = smem[off[2] + n * str[2]];
                            const double w3 = smem[off[3] + n * str[3]], w4 = smem[off[4] + n * str[4]];
                            WfL[n] = face3(w1, w2, w3, dxd, 1, lim);
                            WfR[n] = face3(w2, w3, w4, dxd, -1, lim);
                        }
                        if (lim == 11) {
                            weno3b_faces<M, double>([&](int s, int n) { return (double)smem[off[1 + s] + n * str[1 + s]]; },
                                                    1, WfL);
                            weno3b_faces<M, double>([&](int s, int n) { return (double)smem[off[2 + s] + n * str[2 + s]]; },
                                                    -1, WfR);
                        }
                    } else {
#pragma unroll
                        for (int n = NB0; n < NB1; ++n) {
                            const double w0 = smem[off[0] + n * str[0]], w1 = smem[off[1] + n * str[1]];
                            const double w2 = smem[off[2] + n * str[2]], w3 = smem[off[3] + n * str[3]];
                            const double w4 = smem[off[4] + n * str[4]], w5 = smem[off[5] + n * str[5]];
                            WfL[n] = weno5(w0, w1, w2, w3, w4, 1);
                            WfR[n] = weno5(w1, w2, w3, w4, w5, -1);
                        }
                    }
                    M::prim2cons(UL, WfL, a.e, err);
                    M::prim2cons(UR, WfR, a.e, err);
                    if constexpr (NPH && SCHEME != 6) if (SCHEME != 2 || a.muscl != 11) {
                        // N-phase WENO5 / three-cell schemes: the consistent limiter about the stencil
                        // centres f-1 and f (WENO5B bounds its face values instead)
                        M::consistent_limit(UL, smem + off[2], str[2], dxd, 1, a.e, err);
                        M::consistent_limit(UR, smem + off[3], str[3], dxd, -1, a.e, err);
                    }
                    if constexpr (SXN && SCHEME == 2) if (a.muscl >= 1 && a.muscl < 10) {
                        // N-phase six-equation: the consistent limiter after MUSCL only
                        M::consistent_limit(UL, smem + off[2], str[2], dxd, 1, a.e, err);
                        M::consistent_limit(UR, smem + off[3], str[3], dxd, -1, a.e, err);
                    }
                }
                if constexpr (PFX) {
                    pf_face_fluxes<M, MIX>(F, fnc, UL, UR, pf_face_gq(a, d, gi, gj, gk), a.e, a.pf_phasic, a.pf_hll,
                                           err);
                    cm = 0.0;
                } else {
                    riemann<M>(a.riemann, F, fnc, cm, UL, UR, a.e, d, a.id_k, err);
                }
            } else {
                float wL[N], wR[N];
                if (thinc_face) {
                    M::cons2prim_f32(wL, UL, a.e);
                    M::cons2prim_f32(wR, UR, a.e);
                } else {
                    if constexpr (SCHEME == 6 && (NPH || SXN)) {
                        auto rl = [&](int k, int s) { return (float)smem[off[s] + (M::IR + k) * str[s]]; };
                        auto al_ = [&](int k, int s) { return (float)smem[off[s] + (M::IA + k) * str[s]]; };
                        bounded_phases<M::NP, 5, float>(rl, al_, 1, wL + M::IR, wL + M::IA);
                        auto rr = [&](int k, int s) { return (float)smem[off[s + 1] + (M::IR + k) * str[s + 1]]; };
                        auto ar_ = [&](int k, int s) { return (float)smem[off[s + 1] + (M::IA + k) * str[s + 1]]; };
                        bounded_phases<M::NP, 5, float>(rr, ar_, -1, wR + M::IR, wR + M::IA);
                    } else if constexpr (SCHEME == 6) {
                        float r1[6], r2[6], al[6];
#pragma unroll
                        for (int s = 0; s < 6; ++s) {
                            r1[s] = smem[off[s]];
                            r2[s] = smem[off[s] + str[s]];
                            al[s] = smem[off[s] + M::IA * str[s]];
                        }
                        weno5b_masses_f32(r1, r2, al, 1, wL[0], wL[1], wL[M::IA]);
                        weno5b_masses_f32(r1 + 1, r2 + 1, al + 1, -1, wR[0], wR[1], wR[M::IA]);
                    }
                    if constexpr (SCHEME == 2) {
                        const int lim = a.muscl;
#pragma unroll
                        for (int n = 0; n < N; ++n) {
                            const float w1 = smem[off[1] + n * str[1]], w2 = smem[off[2] + n * str[2]];
                            const float w3 = smem[off[3] + n * str[3]], w4 = smem[off[4] + n * str[4]];
                            wL[n] = face3_f32(w1, w2, w3, 1, lim);
                            wR[n] = face3_f32(w2, w3, w4, -1, lim);
                        }
                        if (lim == 11) {
                            weno3b_faces<M, float>([&](int s, int n) { return (float)smem[off[1 + s] + n * str[1 + s]]; },
                                                   1, wL);
                            weno3b_faces<M, float>([&](int s, int n) { return (float)smem[off[2 + s] + n * str[2 + s]]; },
                                                   -1, wR);
                        }
                    } else {
#pragma unroll
                        for (int n = NB0; n < NB1; ++n) {
                            const float w0 = smem[off[0] + n * str[0]], w1 = smem[off[1] + n * str[1]];
                            const float w2 = smem[off[2] + n * str[2]], w3 = smem[off[3] + n * str[3]];
                            const float w4 = smem[off[4] + n * str[4]], w5 = smem[off[5] + n * str[5]];
                            wL[n] = weno5_f32(w0, w1, w2, w3, w4, 1);
                            wR[n] = weno5_f32(w1, w2, w3, w4, w5, -1);
                        }
                    }
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        WfL[n] = wL[n];
                        WfR[n] = wR[n];
                    }
                    M::prim2cons(UL, WfL, a.e, err);
                    M::prim2cons(UR, WfR, a.e, err);
                    if constexpr (NPH && SCHEME != 6) if (SCHEME != 2 || a.muscl != 11) {
                        M::consistent_limit(UL, smem + off[2], str[2], dxd, 1, a.e, err);
                        M::consistent_limit(UR, smem + off[3], str[3], dxd, -1, a.e, err);
                    }
                    if constexpr (SXN && SCHEME == 2) if (a.muscl >= 1 && a.muscl < 10) {
                        M::consistent_limit(UL, smem + off[2], str[2], dxd, 1, a.e, err);
                        M::consistent_limit(UR, smem + off[3], str[3], dxd, -1, a.e, err);
                    }
                }
                if constexpr (NPH || SXN) {
                    // N-phase models: FP32 reconstruction, FP64 limiter and Riemann solver
                    riemann<M>(a.riemann, F, fnc, cm, UL, UR, a.e, d, a.id_k, err);
                } else {
                    float cmf;
                    if constexpr (PFX) {
                        pf_face_fluxes<M, MIX>(F, fnc, UL, UR, pf_face_gq(a, d, gi, gj, gk), a.e, a.pf_phasic,
                                               a.pf_hll, err);
                        cmf = 0.0f;
                    } else if (a.riemann != 2) {
                        llf_hll_mixed<M>(a.riemann, F, fnc, cmf, UL, UR, wL, wR, a.e, d, a.id_k);
                    } else if constexpr (M::KIND == kModelFive) {
                        fiveeq_hllc_mixed<D>(F, fnc, cmf, UL, UR, wL, wR, a.e, d, a.id_k);
                    } else {
                        sixeq_hllc_mixed<D>(F, fnc, cmf, UL, UR, wL, wR, a.e, d);
                    }
                    cm = cmf;
                }
            }
#pragma unroll
            for (int n = 0; n < N; ++n) Fb[n * FMAX + f] = F[n];
#pragma unroll
            for (int c = 0; c < NC; ++c) Fb[(N + c) * FMAX + f] = fnc[c];
            const int gd = (d == 0) ? gi : (d == 1 ? gj : gk);
            const int nd = (d == 0) ? g.n[0] : (d == 1 ? g.n[1] : g.n[2]);
            if (fd < TS && gd < nd) cmax_local = dmax(cm, cmax_local);
        }
        __syncthreads();

        // 2c. divergence contribution of direction d: (F+ - F-)/dx as the reference divides (FP64 form);
        // times the reciprocal of dx in the mixed form (an FP64 division per term dominates otherwise)
        const double idxd = 1.0 / dxd;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int l = tid + r * NT;
            if (l < CELLS) {
                const int lx = l % TX, ly = (l / TX) % TY, lz = l / (TX * TY);
                // low and high faces of the cell in the enumeration of 2b
                int fl, fh;
                if (d == 0) { fl = lx + EF * (ly + TS * lz); fh = fl + 1; }
                else if (d == 1) { fl = lx + TS * (ly + EF * lz); fh = fl + TS; }
                else { fl = lx + TS * (ly + TS * lz); fh = fl + TS * TS; }
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    const double df = Fb[c * FMAX + fh] - Fb[c * FMAX + fl];
                    const double tt = MIX ? df * idxd : df / dxd;
                    acc[r][c] = (d == 0) ? tt : acc[r][c] + tt;
                }
            }
        }
        // no barrier here: the next direction's halo pass writes only the halo slabs, which this
        // direction's faces finished reading before the barrier above, and its faces overwrite the
        // face buffer only after the barrier that follows that halo pass
    }

    // 3. epilogue
    if (a.mode != kModeCmax) {
        double dt = 0.0, ca = 1.0, cb = 0.0, cd = 1.0;
        if (a.mode == kModeStage) {
            dt = *a.dt;
            if (a.stage == 1) { ca = 0.25; cb = 0.75; cd = 0.25; }
            else if (a.stage == 2) { ca = 2.0 / 3.0; cb = 1.0 / 3.0; cd = 2.0 / 3.0; }
        }
        const double sdt = cd * dt;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int l = tid + r * NT;
            if (l >= CELLS) continue;
            const int lx = l % TX, ly = (l / TX) % TY, lz = l / (TX * TY);
            const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
            if (i >= g.n[0] || j >= g.n[1] || k >= g.n[2]) continue;
            double W[N], L[N];
            const long long q = g.at(i, j, k);
            double Us[N];
            load_cons<M>(Us, a.Us, g, q);
            if constexpr (MIX) {
                // masses and volume fraction exactly from the conserved state (FP64); the pressures
                // of the non-conservative terms from the FP32 tile
#pragma unroll
                for (int n = 0; n < N; ++n) W[n] = Pint[n * CSTR + l];
                if constexpr (NPH || SXN) {
#pragma unroll
                    for (int k = 0; k < M::NP; ++k) {
                        W[M::IR + k] = Us[M::IR + k];
                        W[M::IA + k] = Us[M::IA + k];
                    }
                } else {
                    W[0] = Us[0];
                    W[1] = Us[1];
                    W[M::IA] = Us[M::IA];
                }
            } else {
#pragma unroll
                for (int n = 0; n < N; ++n) W[n] = Pint[n * CSTR + l];
            }
#pragma unroll
            for (int n = 0; n < N; ++n) L[n] = -acc[r][n];
            if constexpr (PFX) {
                if constexpr (M::KIND == kModelSix) {
                    // six-equation: the phase-energy exchange of the regularisation fluxes,
                    // u . (J_k rho_k . grad u) = div(J_k rho_k EK) - EK div(J_k rho_k)
                    // (include/Operators_Compressible6Eq_PhaseField/FVM_PhaseField_SurfaceIntegralNC_Compressible6Eq_PhaseField.H:15-85)
                    const double a1r1 = W[0], a2r2 = W[1];
                    const double rho = a1r1 + a2r2;
                    const double EK = 0.5 * ksum<D>(W + 2);
                    const double vg1 = acc[r][N + 2] - EK * acc[r][N];
                    const double vg2 = acc[r][N + 3] - EK * acc[r][N + 1];
                    const double x = (a1r1 / rho) * vg2 - (a2r2 / rho) * vg1;
                    L[M::IE1] = L[M::IE1] + x;
                    L[M::IE2] = L[M::IE2] + (-x);
                }
                // the five-equation model has no Phase-Field non-conservative terms
                // (include/Operators_Compressible5Eq_PhaseField/FVM_PhaseField_SurfaceIntegralNC_Compressible5Eq_PhaseField.H)
            } else if constexpr (M::KIND == kModelFive) {
                // five-equation: alpha1 += phi1 (1 + K1) div u*
                const double fac = M::kapila_factor(W, W, a.e, a.id_k, err);
                L[M::IA] = L[M::IA] + fac * acc[r][N];
            } else if constexpr (NPH) {
                // N-phase five-equation: alpha_k += phi_k (1 + K_k) div u*
                double fac[M::NP];
                M::kapila_factors(fac, W, a.e, a.id_k, err);
#pragma unroll
                for (int k = 0; k < M::NP; ++k) L[M::IA + k] = L[M::IA + k] + fac[k] * acc[r][N];
            } else if constexpr (SXN) {
                // N-phase six-equation: alpha_k += alpha_k div u*, alpha_k rho_k e_k -= alpha_k p_k div u*
                // (FVM_SurfaceIntegralNC_Compressible6Eq_IE_NPhase.H; acc holds +div u*, the reference
                // subtracts alpha_k times its negative)
                const double divv = acc[r][N];
#pragma unroll
                for (int k = 0; k < M::NP; ++k) {
                    L[M::IA + k] = L[M::IA + k] + W[M::IA + k] * divv;
                    L[M::IP + k] = L[M::IP + k] - W[M::IP + k] * divv;
                }
            } else {
                // six-equation: phase energy exchange and alpha1 div u (FVM_SurfaceIntegralNC_Compressible6Eq.H)
                const double divv = acc[r][N], dva1 = acc[r][N + 1], dva2 = acc[r][N + 2];
                const double a1r1 = W[0], a2r2 = W[1];
                const double rho = a1r1 + a2r2;
                const double vg1 = dva1 - W[M::IE1] * divv;
                const double vg2 = dva2 - W[M::IE2] * divv;
                const double x = (a2r2 / rho) * vg1 - (a1r1 / rho) * vg2;
                L[M::IE1] = L[M::IE1] + x;
                L[M::IE2] = L[M::IE2] + (-x);
                L[M::IA] = L[M::IA] + W[M::IA] * divv;
            }
            double out[N];
            if (a.mode == kModeDudt) {
#pragma unroll
                for (int n = 0; n < N; ++n) out[n] = L[n];
            } else {
                if (a.stage == 0) {
#pragma unroll
                    for (int n = 0; n < N; ++n) out[n] = 1.0 * Us[n] + sdt * L[n];
                } else {
                    double U0[N];
                    load_cons<M>(U0, a.U0, g, q);
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        double v = ca * Us[n] + cb * U0[n];
                        out[n] = v + sdt * L[n];
                    }
                }
                if constexpr (M::KIND == kModelSix) {
                    if (a.relax) relax_pressure<D, MIX>(out, a.e, a.trace, err);
                } else if constexpr (SXN) {
                    if (a.relax) M::relax(out, a.e, a.trace, err);
                }
                bool bad = false;
#pragma unroll
                for (int n = 0; n < N; ++n) bad |= isnan(out[n]);
                if (bad) flag_error(err, COMPAS_B200_ERR_NAN);
            }
#pragma unroll
            for (int n = 0; n < N; ++n) a.Uout[n * g.S + q] = out[n];
        }
    }

    // CTA max of the face wave speeds -> one atomic
    if (a.cmax) {
        double v = cmax_local;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        __shared__ double wmax[32];
        const int w = tid >> 5, lane = tid & 31;
        if (lane == 0) wmax[w] = v;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int q = 0; q < (NT + 31) / 32; ++q) m = dmax(m, wmax[q]);
            // non-negative doubles order like their bit patterns; a NaN speed propagates as the max
            atomicMax(a.cmax, (unsigned long long)__double_as_longlong(m));
        }
    }
}

// One box: one CTA per tile.
template <class M, int SCHEME, bool MIX, int VAR, int TX, int TY, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(StageArgs a) {
    if (a.done && *a.done) return;
    extern __shared__ double smem_d[];
    stage_tile<M, SCHEME, MIX, VAR, TX, TY, TZ, NT>(a, a.tile_base + blockIdx.x, smem_d);
}

// One box with the halo slabs staged by TMA (the tensor maps of a.Us are kernel parameters).
template <class M, int SCHEME, bool MIX, int TX, int TY, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_kernel_tma(StageArgs a, const __grid_constant__ TmaMaps tm) {
    if (a.done && *a.done) return;
    extern __shared__ __align__(128) double smem_d[];
    stage_tile<M, SCHEME, MIX, kVarTma, TX, TY, TZ, NT>(a, a.tile_base + blockIdx.x, smem_d, &tm);
}

// ------------------------------------------------------------------------------------------------
// Box list: many boxes (independent cases of uneven size, or the boxes of a level) in one
// persistent launch. The list, its tile prefix sums and its length live in device memory, so a
// captured CUDA graph stays valid while boxes are added or removed between launches.
// ------------------------------------------------------------------------------------------------
struct BoxDesc {
    Grid g;
    Eos e;
    double* U[3];                 // U^n, U^(1), U^(2) of the box (stage s reads U[s], writes U[(s+1)%3])
    const double* dt;             // the box's time step (device)
    const int* done;              // the box's no-op flag (device)
    unsigned long long* cmax;     // the box's wave-speed accumulator (device)
    unsigned int* err;            // the box's status word (device)
    int lo_bc[3], hi_bc[3];
    int id_k;
    int relax;
    int riemann;                  // Physics.RiemannSolver of the box's case (0 LLF, 1 HLL, 2 HLLC)
    int muscl;                    // three-cell scheme code of the box's case (StageArgs::muscl)
    double trace;
    int tiles;                    // tiles of the box for the kernel's tile shape
    long long ghosts;             // ghost cells of one array of the box
    double* out_last;             // output of the last stage (nullptr: in place over U[0])
};

struct ListArgs {
    const BoxDesc* boxes;
    const int* nbox;              // number of boxes (device)
    const int* tile_off;          // exclusive prefix sums of BoxDesc::tiles, nbox + 1 entries
    int mode;
    int stage;
    int order;                    // tile traversal order inside each box (tile_coords)
};

__device__ __forceinline__ int find_box(const int* off, int nb, int w) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= w) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The arguments of the current tile's box live in shared memory: the tile code reads them where it
// needs them (as the single-box kernel reads its parameters from the constant bank) instead of
// holding a per-thread copy of the grid and EOS in registers.
template <class M, int SCHEME, bool MIX, int TX, int TY, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_list_kernel(ListArgs L) {
    extern __shared__ double smem_d[];
    __shared__ StageArgs sa;
    static_assert(sizeof(Grid) % 8 == 0 && sizeof(Eos) % 8 == 0, "word copies of the grid and EOS");
    constexpr int GW = sizeof(Grid) / 8, EW = sizeof(Eos) / 8;
    static_assert(GW + EW <= NT, "one word per thread");
    const int nb = *L.nbox;
    if (nb <= 0) return;
    const int total = L.tile_off[nb];
    const int tid = threadIdx.x;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        const int b = find_box(L.tile_off, nb, w);
        const BoxDesc& B = L.boxes[b];
        if (*B.done) continue;
        __syncthreads();  // the previous tile's readers of shared memory (and of sa) are done
        if (tid < GW) {
            reinterpret_cast<unsigned long long*>(&sa.g)[tid] = reinterpret_cast<const unsigned long long*>(&B.g)[tid];
        } else if (tid < GW + EW) {
            reinterpret_cast<unsigned long long*>(&sa.e)[tid - GW] =
                reinterpret_cast<const unsigned long long*>(&B.e)[tid - GW];
        } else if (tid == GW + EW) {
            sa.mode = L.mode;
            sa.stage = L.stage;
            sa.Us = B.U[L.stage];
            sa.U0 = B.U[0];
            sa.Uout = (L.stage == 2 && B.out_last) ? B.out_last : B.U[(L.stage + 1) % 3];
            sa.dt = B.dt;
            sa.done = B.done;
            sa.cmax = B.cmax;
            sa.err = B.err;
            sa.id_k = B.id_k;
            sa.relax = B.relax;
            sa.trace = B.trace;
            sa.order = L.order;
            sa.tile_base = 0;
            sa.tile_count = 0;
            sa.pf_phasic = 0;
            sa.pf_hll = 0;
            sa.muscl = B.muscl;
            sa.riemann = B.riemann;
            for (int d = 0; d < 3; ++d) sa.gq[d] = nullptr;
        }
        __syncthreads();
        stage_tile<M, SCHEME, MIX, kVarPlain, TX, TY, TZ, NT>(sa, w - L.tile_off[b], smem_d);
    }
}

}  // namespace compas
