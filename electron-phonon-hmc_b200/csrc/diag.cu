// Diagnostics: a count of this library's kernel launches and a CUDA-core FMA
// throughput probe (FP32 / FP64), the roofline denominator for the stencil
// kernels, which run on the CUDA cores rather than HBM- or tensor-core-bound.
#include "ephmc_internal.cuh"

#include <atomic>

namespace ephmc {
namespace {
std::atomic<unsigned long long> g_launches{0};
}
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace ephmc

using namespace ephmc;

namespace ephmc_diag {

// 8 independent FMA chains per thread, unrolled; result folded so the compiler keeps it.
template <typename T>
__global__ void k_fma_probe(T *out, int iters, T a, T b) {
    T v0 = threadIdx.x * (T)1e-3, v1 = v0 + (T)1, v2 = v0 + (T)2, v3 = v0 + (T)3;
    T v4 = v0 + (T)4, v5 = v0 + (T)5, v6 = v0 + (T)6, v7 = v0 + (T)7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            v0 = fma(v0, a, b);
            v1 = fma(v1, a, b);
            v2 = fma(v2, a, b);
            v3 = fma(v3, a, b);
            v4 = fma(v4, a, b);
            v5 = fma(v5, a, b);
            v6 = fma(v6, a, b);
            v7 = fma(v7, a, b);
        }
    }
    const T s = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
    if (s == (T)-12345.678) out[blockIdx.x] = s;
}

template <typename T>
int probe(float *tflops) {
    int dev = 0, sms = 0;
    EPHMC_CUDA(cudaGetDevice(&dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T *out = nullptr;
    EPHMC_CUDA(cudaMalloc(&out, sizeof(T) * 4096));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_probe<T><<<blocks, threads>>>(out, 64, (T)0.999, (T)1e-4);  // warm-up
    cudaEventRecord(e0);
    k_fma_probe<T><<<blocks, threads>>>(out, iters, (T)0.999, (T)1e-4);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    EPHMC_CUDA(cudaGetLastError());
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = (float)(flops / (ms * 1e-3) / 1e12);
    return EPHMC_OK;
}

}  // namespace ephmc_diag

using ephmc_diag::probe;

extern "C" {

EPHMC_API unsigned long long ephmc_launch_count(void) { return g_launches.load(); }

EPHMC_API int ephmc_measure_fma_peak(int fp64, float *tflops) {
    if (!tflops) return EPHMC_ERR_ARG;
    return fp64 ? probe<double>(tflops) : probe<float>(tflops);
}

}  // extern "C"
