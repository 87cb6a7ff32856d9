// Throughput probes of the FP32 and FP64 FMA pipes, the denominators of the compute roofline that
// bench.py reports beside the HBM one (the stage kernels are instruction-bound, not HBM-bound).
// Every thread runs eight independent FMA chains, the grid fills every SM at full occupancy, so the
// measured rate is the pipe's sustained FMA rate at the clock the GPU runs at; one FMA counts as two
// floating-point operations.
#include <cuda_runtime.h>

#include "compas_b200.h"

namespace {

__device__ double g_peak_sink;

template <class T>
__global__ void __launch_bounds__(256) fma_peak_kernel(int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = (T)(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += x[c];
    if (s == (T)-1.2345) g_peak_sink = (double)s;  // never true for these inputs; keeps the chains live
}

}  // namespace

extern "C" int compas_b200_fma_peak(int fp64, int iters, double* flops_per_s, void* stream) {
    if (!flops_per_s || iters <= 0) return COMPAS_B200_EARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return COMPAS_B200_ECUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return COMPAS_B200_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const int threads = 256, blocks = sms * 8;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return COMPAS_B200_ECUDA;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return COMPAS_B200_ECUDA;
    }
    // warm-up launch, then the timed one
    for (int rep = 0; rep < 2; ++rep) {
        if (rep == 1) cudaEventRecord(e0, st);
        if (fp64) fma_peak_kernel<double><<<blocks, threads, 0, st>>>(iters, 0.999999, 1e-7);
        else fma_peak_kernel<float><<<blocks, threads, 0, st>>>(iters, 0.999999f, 1e-7f);
    }
    cudaEventRecord(e1, st);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess || cudaGetLastError() != cudaSuccess || ms <= 0.0f) return COMPAS_B200_ECUDA;
    *flops_per_s = 2.0 * 8.0 * (double)iters * (double)threads * (double)blocks / (ms * 1e-3);
    return COMPAS_B200_OK;
}
