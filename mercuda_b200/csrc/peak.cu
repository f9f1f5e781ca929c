// FP64 issue-rate probe: the denominator of the FP64 roofline. Every thread
// runs eight independent dependent chains of fma() (2 FLOP each) so that the
// FP64 pipe, not latency, bounds the loop; the grid covers every SM.
#include <cuda_runtime.h>

#include "../../include/mercury_b200.h"

namespace {
__global__ void __launch_bounds__(256) fma_chains(double* sink, int iters, double a, double b) {
    double r[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = a + (threadIdx.x + k) * 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = fma(r[k], b, a);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += r[k];
    if (s == 1.2345) sink[blockIdx.x] = s;  // keeps the chains live, never true in practice
}
}  // namespace

extern "C" int mercury_b200_fp64_peak(double* tflops, double* ms) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double) * blocks) != cudaSuccess) return 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chains<<<blocks, threads>>>(sink, iters, 0.5, 0.999999);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fma_chains<<<blocks, threads>>>(sink, iters, 0.5, 0.999999);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (t < best) best = t;
    }
    const double flop = 2.0 * 8.0 * (double)iters * threads * blocks;
    *tflops = flop / (best * 1e-3) / 1e12;
    if (ms) *ms = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
