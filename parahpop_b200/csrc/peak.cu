// FMA-throughput microbenchmark: the FP64 / FP32 roofline denominator for the
// step kernel, measured on the device the library runs on.  Each thread runs
// eight independent FMA chains so the pipes, not latency, bound the loop.
#include <cuda_runtime.h>

#include "../../include/parahpop.h"

namespace {
template <typename T>
__global__ void fmaPeakKernel(T* out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == (T)12345.678) out[threadIdx.x] = s;  // keeps the chains alive
}

template <typename T>
double measure(int device) {
    cudaSetDevice(device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    T* out = nullptr;
    if (cudaMalloc(&out, 1024 * sizeof(T)) != cudaSuccess) return -1.0;
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        fmaPeakKernel<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
        if (rep > 0 && ms > 0) best = best > flops / (ms * 1e-3) ? best : flops / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return cudaGetLastError() == cudaSuccess ? best * 1e-12 : -1.0;
}
}  // namespace

extern "C" int phop_fma_peak(int device, double* fp64_tflops, double* fp32_tflops) {
    if (fp64_tflops) *fp64_tflops = measure<double>(device);
    if (fp32_tflops) *fp32_tflops = measure<float>(device);
    return (fp64_tflops && *fp64_tflops < 0) || (fp32_tflops && *fp32_tflops < 0) ? 1 : 0;
}
