// One (precision, time-grid mode) family of step-kernel instantiations.  The
// build compiles this file four times with PHOP_T = double | float and
// PHOP_SG = 1 (shared time grid) | 0 (per-object time), in parallel.
#include <cuda_runtime.h>

#include "nrlmsise00.cuh"
#include "propagate.cuh"
#include "propagate_impl.cuh"

#ifndef PHOP_T
#define PHOP_T double
#endif
#ifndef PHOP_SG
#define PHOP_SG 1
#endif
#ifndef PHOP_SUFFIX
#define PHOP_SUFFIX f64_grid
#endif
#define PHOP_CAT2(a, b) a##b
#define PHOP_CAT(a, b) PHOP_CAT2(a, b)

namespace phop {

template <int L>
static cudaError_t launchOne(const StepParams& p, int ctas, int threads, int smem, cudaStream_t stream) {
    auto k = propagateKernel<L, PHOP_T, (bool)PHOP_SG>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
    }
    k<<<ctas, threads, smem, stream>>>(p);
    return cudaGetLastError();
}

template <int L>
static int occupancyOne(int threads, int smem) {
    int n = 0;
    auto k = propagateKernel<L, PHOP_T, (bool)PHOP_SG>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem);
    return n;
}

cudaError_t PHOP_CAT(launchPropagate_, PHOP_SUFFIX)(const StepParams& p, size_t paramsBytes, int lanes, int ctas,
                                                    int threads, int smem, cudaStream_t stream) {
    if (paramsBytes != sizeof(StepParams)) return cudaErrorInvalidValue;  // objects built from different headers
    switch (lanes) {
        case 1: return launchOne<1>(p, ctas, threads, smem, stream);
        case 2: return launchOne<2>(p, ctas, threads, smem, stream);
        case 4: return launchOne<4>(p, ctas, threads, smem, stream);
        case 8: return launchOne<8>(p, ctas, threads, smem, stream);
        case 16: return launchOne<16>(p, ctas, threads, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

int PHOP_CAT(occupancy_, PHOP_SUFFIX)(int lanes, int threads, int smem) {
    switch (lanes) {
        case 1: return occupancyOne<1>(threads, smem);
        case 2: return occupancyOne<2>(threads, smem);
        case 4: return occupancyOne<4>(threads, smem);
        case 8: return occupancyOne<8>(threads, smem);
        case 16: return occupancyOne<16>(threads, smem);
        default: return 0;
    }
}

}  // namespace phop
