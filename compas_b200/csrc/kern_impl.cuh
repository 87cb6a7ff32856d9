// Instantiation and launch of the stage kernels of one model and dimension (included once by each
// kern_*.cu translation unit).
#pragma once

#include <algorithm>
#include <type_traits>

#include "launch.h"
#include "stage_kernel.cuh"

namespace compas {

// Launch shapes of the stage kernel (threads per CTA, CTAs per SM) among which the autotuner picks;
// the tile is 8^3 in 3D and 16^2 in 2D for every shape. The register budget is set per SM
// sub-partition (16384 registers each, warps dealt round-robin): in 3D, 6 warps at 2 CTAs/SM get
// 168 registers per thread, 8 warps 128, 9 warps 112; in 2D, 272 threads at 2 CTAs/SM get 96, at 1
// CTA/SM 232, 136 threads at 4 CTAs/SM 120. Every shape covers the 576 (3D) or 272 (2D) faces of a
// direction in whole rounds or nearly so. Shape 0 is the default when tuning is off.
template <int D, int S>
struct ShapeParams;
template <> struct ShapeParams<3, 0> { static constexpr int NT = 192, MINB = 2; };
template <> struct ShapeParams<3, 1> { static constexpr int NT = 256, MINB = 2; };
template <> struct ShapeParams<3, 2> { static constexpr int NT = 288, MINB = 2; };
template <> struct ShapeParams<2, 0> { static constexpr int NT = 272, MINB = 2; };
template <> struct ShapeParams<2, 1> { static constexpr int NT = 272, MINB = 1; };
template <> struct ShapeParams<2, 2> { static constexpr int NT = 136, MINB = 4; };

template <class M, int S = 0>
struct LaunchShape {
    static constexpr int TS = (M::D == 2) ? kTile2 : kTile3;
    static constexpr int TZ = (M::D == 2) ? 1 : TS;
    static constexpr int NT = ShapeParams<M::D, S>::NT;
    static constexpr int MINB = ShapeParams<M::D, S>::MINB;
};

// One CTA per tile of the box.
template <class M, int SCHEME, bool MIX, int VAR, int SH>
static cudaError_t launch_stage_v(const StageArgs& a, cudaStream_t st) {
    using S = LaunchShape<M, SH>;
    using T = TileShape<M, S::TS, S::TS, S::TZ, typename std::conditional<MIX, float, double>::type, false,
                        VAR == kVarPhaseField>;
    auto kern = stage_kernel<M, SCHEME, MIX, VAR, S::TS, S::TS, S::TZ, S::NT, S::MINB>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const long long tiles = a.tile_count > 0 ? (long long)a.tile_count
                                             : (long long)((a.g.n[0] + S::TS - 1) / S::TS) *
                                                   ((a.g.n[1] + S::TS - 1) / S::TS) * ((a.g.n[2] + S::TZ - 1) / S::TZ);
    kern<<<(unsigned)tiles, S::NT, T::SMEM, st>>>(a);
    return cudaGetLastError();
}

// One box with the y/z halo slabs staged by TMA (3D mixed form; the maps describe a.Us).
template <class M, int SCHEME, int SH>
static cudaError_t launch_stage_tma(const StageArgs& a, const TmaMaps& tm, cudaStream_t st) {
    using S = LaunchShape<M, SH>;
    using T = TileShape<M, S::TS, S::TS, S::TZ, float, true>;
    auto kern = stage_kernel_tma<M, SCHEME, true, S::TS, S::TS, S::TZ, S::NT, S::MINB>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const long long tiles = a.tile_count > 0 ? (long long)a.tile_count
                                             : (long long)((a.g.n[0] + S::TS - 1) / S::TS) *
                                                   ((a.g.n[1] + S::TS - 1) / S::TS) * ((a.g.n[2] + S::TZ - 1) / S::TZ);
    kern<<<(unsigned)tiles, S::NT, T::SMEM, st>>>(a, tm);
    return cudaGetLastError();
}

template <class M, int SCHEME, bool MIX>
static cudaError_t launch_stage_var(const KernelChoice& k, const StageArgs& a, cudaStream_t st, const TmaMaps* tm) {
    if constexpr (SCHEME == 2) {
        // GODUNOV / MUSCL: the plain right-hand side, ordinary halo loads (the tuner's TMA candidate
        // runs this form too)
        if (k.phase_field || k.thinc) return cudaErrorNotSupported;
        switch (k.shape) {
            case 1: return launch_stage_v<M, 2, MIX, kVarPlain, 1>(a, st);
            case 2: return launch_stage_v<M, 2, MIX, kVarPlain, 2>(a, st);
            default: return launch_stage_v<M, 2, MIX, kVarPlain, 0>(a, st);
        }
    } else {
    if constexpr (M::D == 3 && MIX && M::KIND != kModelFiveN && M::KIND != kModelSixN) {
        if (tm && tm->valid && !k.thinc && !k.phase_field) {
            switch (k.shape) {
                case 1: return launch_stage_tma<M, SCHEME, 1>(a, *tm, st);
                case 2: return launch_stage_tma<M, SCHEME, 2>(a, *tm, st);
                default: return launch_stage_tma<M, SCHEME, 0>(a, *tm, st);
            }
        }
    }
    if constexpr (M::KIND == kModelFiveN || M::KIND == kModelSixN) {
        // FIVEEQS_NPHASE, SIXEQS_IE_NPHASE: the plain hyperbolic right-hand side only
        if (k.phase_field || k.thinc) return cudaErrorNotSupported;
    } else {
        // the THINC and Phase-Field variants run at shape 0
        if (k.phase_field) return launch_stage_v<M, SCHEME, MIX, kVarPhaseField, 0>(a, st);
        if (k.thinc) return launch_stage_v<M, SCHEME, MIX, kVarThinc, 0>(a, st);
    }
    switch (k.shape) {
        case 1: return launch_stage_v<M, SCHEME, MIX, kVarPlain, 1>(a, st);
        case 2: return launch_stage_v<M, SCHEME, MIX, kVarPlain, 2>(a, st);
        default: return launch_stage_v<M, SCHEME, MIX, kVarPlain, 0>(a, st);
    }
    }
}

// The kernels of one precision form (MIX); the two forms are separate translation units (built in
// parallel).
template <class M, bool MIX>
static cudaError_t launch_stage_m(const KernelChoice& k, const StageArgs& a, cudaStream_t st, const TmaMaps* tm) {
    if (k.limiter < 5) return launch_stage_var<M, 2, MIX>(k, a, st, tm);  // GODUNOV / MUSCL / WENO3 family
    return (k.limiter == 6) ? launch_stage_var<M, 6, MIX>(k, a, st, tm) : launch_stage_var<M, 5, MIX>(k, a, st, tm);
}

// Persistent box-list launch: one resident wave of CTAs walks the tiles of every box.
template <class M, int SCHEME, bool MIX, int SH>
static cudaError_t launch_list_v(const ListArgs& L, cudaStream_t st) {
    using S = LaunchShape<M, SH>;
    using T = TileShape<M, S::TS, S::TS, S::TZ, typename std::conditional<MIX, float, double>::type>;
    auto kern = stage_list_kernel<M, SCHEME, MIX, S::TS, S::TS, S::TZ, S::NT, S::MINB>;
    static int grid = 0;
    if (!grid) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, S::NT, T::SMEM)) != cudaSuccess) return e;
        grid = sms * std::max(per, 1);
    }
    kern<<<grid, S::NT, T::SMEM, st>>>(L);
    return cudaGetLastError();
}

template <class M, int SCHEME, bool MIX>
static cudaError_t launch_list_s(const KernelChoice& k, const ListArgs& L, cudaStream_t st) {
    switch (k.shape) {
        case 1: return launch_list_v<M, SCHEME, MIX, 1>(L, st);
        case 2: return launch_list_v<M, SCHEME, MIX, 2>(L, st);
        default: return launch_list_v<M, SCHEME, MIX, 0>(L, st);
    }
}

template <class M, bool MIX>
static cudaError_t launch_list_m(const KernelChoice& k, const ListArgs& L, cudaStream_t st) {
    if (k.limiter < 5) return launch_list_s<M, 2, MIX>(k, L, st);  // GODUNOV / MUSCL / WENO3 family
    return (k.limiter == 6) ? launch_list_s<M, 6, MIX>(k, L, st) : launch_list_s<M, 5, MIX>(k, L, st);
}

}  // namespace compas

// PREC 0: the plain FP64 form (launch_*_<name>_p0), PREC 1: the mixed form (launch_*_<name>_p1).
#define COMPAS_DEFINE_LAUNCHERS(name, Model, PREC)                                                   \
    namespace compas {                                                                              \
    cudaError_t launch_stage_##name##_p##PREC(const KernelChoice& k, const StageArgs& a, cudaStream_t st, \
                                              const TmaMaps* tm) {                                  \
        return launch_stage_m<Model, PREC == 1>(k, a, st, tm);                                      \
    }                                                                                               \
    cudaError_t launch_list_##name##_p##PREC(const KernelChoice& k, const ListArgs& L, cudaStream_t st) { \
        return launch_list_m<Model, PREC == 1>(k, L, st);                                           \
    }                                                                                               \
    }
