// Asynchronous bulk-tensor (TMA) loads of the stage kernel's halo slabs on sm_100a: one thread issues
// cp.async.bulk.tensor copies of a box of the padded state array into shared memory, completion is
// tracked by a CTA mbarrier with a transaction count, and every wait is bounded (a copy that does not
// complete sets a status bit instead of spinning forever). The copies are single-CTA (no multicast).
#pragma once

#include <cuda.h>
#include <cstdint>

namespace compas {

// The two tensor maps of one padded state array (Array4 layout, dims {PX, PY, PZ, N}, FP64): boxes of
// the y-direction halo slabs (10 x 3 x 8 x N) and of the z-direction slabs (10 x 8 x 3 x N) of an 8^3
// tile. valid = 0: no maps (the kernel loads the slabs with ordinary loads).
struct TmaMaps {
    CUtensorMap y;
    CUtensorMap z;
    int valid;
};

constexpr int kTmaBoxX = 10;  // 8 tile cells plus an even-aligned start: x runs from an even index

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory before later async-proxy
// (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One box of a 4D tensor map at coordinates (x, y, z, c) into shared memory at dst (128-byte aligned),
// completing on bar.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z,
                                            int c) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::
            "r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of bar with at most `limit` polls; false if it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit) {
    for (int it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace compas
