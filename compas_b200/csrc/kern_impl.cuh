// Instantiation and launch of the stage kernels of one model and dimension (included once by each
// kern_*.cu translation unit).
#pragma once

#include <algorithm>
#include <type_traits>

#include "launch.h"
#include "stage_kernel.cuh"

// Launch shape of the stage kernel: threads per CTA and CTAs per SM of the 3D (8^3 tile) and 2D
// (16^2 tile) kernels. The register budget is set per SM sub-partition (16384 registers each, warps
// dealt round-robin), so a CTA of 6 warps at 2 CTAs/SM gets 168 registers per thread.
#ifndef COMPAS_NT3
#define COMPAS_NT3 192
#endif
#ifndef COMPAS_MINB3
#define COMPAS_MINB3 2
#endif
#ifndef COMPAS_NT2
#define COMPAS_NT2 272
#endif
#ifndef COMPAS_MINB2
#define COMPAS_MINB2 2
#endif

namespace compas {

template <class M>
struct LaunchShape {
    static constexpr int TS = (M::D == 2) ? kTile2 : kTile3;
    static constexpr int TZ = (M::D == 2) ? 1 : TS;
    static constexpr int NT = (M::D == 2) ? COMPAS_NT2 : COMPAS_NT3;
    static constexpr int MINB = (M::D == 2) ? COMPAS_MINB2 : COMPAS_MINB3;
};

// One CTA per tile of the box.
template <class M, int SCHEME, bool MIX, int VAR>
static cudaError_t launch_stage_v(const StageArgs& a, cudaStream_t st) {
    using S = LaunchShape<M>;
    using T = TileShape<M, S::TS, S::TS, S::TZ, typename std::conditional<MIX, float, double>::type>;
    auto kern = stage_kernel<M, SCHEME, MIX, VAR, S::TS, S::TS, S::TZ, S::NT, S::MINB>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const long long tiles = (long long)((a.g.n[0] + S::TS - 1) / S::TS) * ((a.g.n[1] + S::TS - 1) / S::TS) *
                            ((a.g.n[2] + S::TZ - 1) / S::TZ);
    kern<<<(unsigned)tiles, S::NT, T::SMEM, st>>>(a);
    return cudaGetLastError();
}

template <class M, int SCHEME, bool MIX>
static cudaError_t launch_stage_var(const KernelChoice& k, const StageArgs& a, cudaStream_t st) {
    if constexpr (M::KIND == kModelFiveN) {
        // FIVEEQS_NPHASE: the plain hyperbolic right-hand side only
        if (k.phase_field || k.thinc) return cudaErrorNotSupported;
        return launch_stage_v<M, SCHEME, MIX, kVarPlain>(a, st);
    } else {
        if (k.phase_field) {
            if constexpr (M::KIND == kModelFive) return launch_stage_v<M, SCHEME, MIX, kVarPhaseField>(a, st);
            else return cudaErrorNotSupported;
        }
        if (k.thinc) return launch_stage_v<M, SCHEME, MIX, kVarThinc>(a, st);
        return launch_stage_v<M, SCHEME, MIX, kVarPlain>(a, st);
    }
}

template <class M>
static cudaError_t launch_stage_m(const KernelChoice& k, const StageArgs& a, cudaStream_t st) {
    const bool mix = (k.precision == 1), bounded = (k.limiter == 6);
    if constexpr (M::KIND == kModelFiveN) {
        if (bounded) return cudaErrorNotSupported;
        return mix ? launch_stage_var<M, 5, true>(k, a, st) : launch_stage_var<M, 5, false>(k, a, st);
    } else {
        if (mix) return bounded ? launch_stage_var<M, 6, true>(k, a, st) : launch_stage_var<M, 5, true>(k, a, st);
        return bounded ? launch_stage_var<M, 6, false>(k, a, st) : launch_stage_var<M, 5, false>(k, a, st);
    }
}

// Persistent box-list launch: one resident wave of CTAs walks the tiles of every box.
template <class M, int SCHEME, bool MIX>
static cudaError_t launch_list_v(const ListArgs& L, cudaStream_t st) {
    using S = LaunchShape<M>;
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

template <class M>
static cudaError_t launch_list_m(const KernelChoice& k, const ListArgs& L, cudaStream_t st) {
    if constexpr (M::KIND == kModelFiveN) {
        if (k.limiter == 6) return cudaErrorNotSupported;
        return (k.precision == 1) ? launch_list_v<M, 5, true>(L, st) : launch_list_v<M, 5, false>(L, st);
    } else {
        if (k.precision == 1) return (k.limiter == 6) ? launch_list_v<M, 6, true>(L, st) : launch_list_v<M, 5, true>(L, st);
        return (k.limiter == 6) ? launch_list_v<M, 6, false>(L, st) : launch_list_v<M, 5, false>(L, st);
    }
}

}  // namespace compas

#define COMPAS_DEFINE_LAUNCHERS(name, Model)                                                         \
    namespace compas {                                                                              \
    cudaError_t launch_stage_##name(const KernelChoice& k, const StageArgs& a, cudaStream_t st) {    \
        return launch_stage_m<Model>(k, a, st);                                                     \
    }                                                                                               \
    cudaError_t launch_list_##name(const KernelChoice& k, const ListArgs& L, cudaStream_t st) {      \
        return launch_list_m<Model>(k, L, st);                                                      \
    }                                                                                               \
    }
