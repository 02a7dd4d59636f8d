// NRLMSISE-00 total mass density for arbitrary inputs through the step
// kernel's own per-object path (nrlf::Fast, lane-split as in the kernel):
// the known-answer check of the device model against the reference's
// gtd7d (Nrlmsise00Model.inl:959-1100, switch 9 = -1).
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "nrl_fast.cuh"

namespace phop {

template <int L>
__global__ void nrlDensityBatchKernel(const nrlf::NrlEpochBlock* __restrict__ blocks, const double* __restrict__ in,
                                      int n, double* __restrict__ out) {
    const int lane = (int)(threadIdx.x & 31);
    const int j = lane % L, groupBase = lane - j;
    int o = (int)((blockIdx.x * blockDim.x + threadIdx.x) / L);
    const bool live = o < n;
    if (!live) o = 0;  // keep the groups of a warp converged; results discarded
    const double* v = in + 16 * (size_t)o;
    nrlf::Fast<double> m(blocks[o], v[1]);
    const double rho = m.template density<L>(v[3], v[4], v[2], v[5], j, groupBase);
    if (live && j == 0) out[o] = rho;
}

// inputs: n rows of {doy, sec, alt, g_lat, g_long, lst, f107A, f107, ap, ap_a[0..6]}
void nrlDensityBatch(int device, int64_t n, const double* inputs, int lanes, double* outRho) {
    if (n < 0 || n > (1 << 24)) throw std::runtime_error("n must be in [0, 2^24]");
    if (n > 0 && (!inputs || !outRho)) throw std::runtime_error("null input or output pointer");
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) throw std::runtime_error("lanes must be 1, 2, 4 or 8");
    if (n == 0) return;
    auto check = [](cudaError_t e) {
        if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
    };
    check(cudaSetDevice(device));
    std::vector<nrlf::NrlEpochBlock> blocks((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const double* v = inputs + 16 * i;
        nrlf::nrlSlotBlock((int)v[0], v[7], v[6], v + 9, blocks[(size_t)i]);
        if (!blocks[(size_t)i].valid) throw std::runtime_error("NRLMSISE-00 block construction failed");
    }
    nrlf::NrlEpochBlock* dBlocks = nullptr;
    double *dIn = nullptr, *dOut = nullptr;
    try {
        check(cudaMalloc(&dBlocks, blocks.size() * sizeof(nrlf::NrlEpochBlock)));
        check(cudaMalloc(&dIn, (size_t)n * 16 * sizeof(double)));
        check(cudaMalloc(&dOut, (size_t)n * sizeof(double)));
        check(cudaMemcpy(dBlocks, blocks.data(), blocks.size() * sizeof(nrlf::NrlEpochBlock), cudaMemcpyHostToDevice));
        check(cudaMemcpy(dIn, inputs, (size_t)n * 16 * sizeof(double), cudaMemcpyHostToDevice));
        const int threads = 128;
        const unsigned grid = (unsigned)(((int64_t)n * lanes + threads - 1) / threads);
        switch (lanes) {
            case 1: nrlDensityBatchKernel<1><<<grid, threads>>>(dBlocks, dIn, (int)n, dOut); break;
            case 2: nrlDensityBatchKernel<2><<<grid, threads>>>(dBlocks, dIn, (int)n, dOut); break;
            case 4: nrlDensityBatchKernel<4><<<grid, threads>>>(dBlocks, dIn, (int)n, dOut); break;
            default: nrlDensityBatchKernel<8><<<grid, threads>>>(dBlocks, dIn, (int)n, dOut); break;
        }
        check(cudaGetLastError());
        check(cudaMemcpy(outRho, dOut, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    } catch (...) {
        cudaFree(dBlocks);
        cudaFree(dIn);
        cudaFree(dOut);
        throw;
    }
    cudaFree(dBlocks);
    cudaFree(dIn);
    cudaFree(dOut);
}

}  // namespace phop
