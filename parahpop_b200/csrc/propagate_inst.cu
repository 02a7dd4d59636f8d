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

template <int L, bool PAIR>
static cudaError_t launchOne(const StepParams& p, int ctas, int threads, int smem, cudaStream_t stream) {
    auto k = propagateKernel<L, PHOP_T, (bool)PHOP_SG, PAIR>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
    }
    k<<<ctas, threads, smem, stream>>>(p);
    return cudaGetLastError();
}

template <int L, bool PAIR>
static int occupancyOne(int threads, int smem) {
    int n = 0;
    auto k = propagateKernel<L, PHOP_T, (bool)PHOP_SG, PAIR>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem);
    return n;
}

cudaError_t PHOP_CAT(launchPropagate_, PHOP_SUFFIX)(const StepParams& p, size_t paramsBytes, int lanes, int ctas,
                                                    int threads, int smem, cudaStream_t stream) {
    if (paramsBytes != sizeof(StepParams)) return cudaErrorInvalidValue;  // objects built from different headers
    // lane-group pairs at up to four lanes only (slower at eight and sixteen)
    if (p.pairSh) {
        switch (lanes) {
            case 1: return launchOne<1, true>(p, ctas, threads, smem, stream);
            case 2: return launchOne<2, true>(p, ctas, threads, smem, stream);
            case 4: return launchOne<4, true>(p, ctas, threads, smem, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (lanes) {
        case 1: return launchOne<1, false>(p, ctas, threads, smem, stream);
        case 2: return launchOne<2, false>(p, ctas, threads, smem, stream);
        case 4: return launchOne<4, false>(p, ctas, threads, smem, stream);
        case 8: return launchOne<8, false>(p, ctas, threads, smem, stream);
        case 16: return launchOne<16, false>(p, ctas, threads, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

int PHOP_CAT(occupancy_, PHOP_SUFFIX)(int lanes, int pair, int threads, int smem) {
    if (pair) {
        switch (lanes) {
            case 1: return occupancyOne<1, true>(threads, smem);
            case 2: return occupancyOne<2, true>(threads, smem);
            case 4: return occupancyOne<4, true>(threads, smem);
            default: return 0;
        }
    }
    switch (lanes) {
        case 1: return occupancyOne<1, false>(threads, smem);
        case 2: return occupancyOne<2, false>(threads, smem);
        case 4: return occupancyOne<4, false>(threads, smem);
        case 8: return occupancyOne<8, false>(threads, smem);
        case 16: return occupancyOne<16, false>(threads, smem);
        default: return 0;
    }
}

}  // namespace phop
