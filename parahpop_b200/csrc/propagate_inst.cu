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

// one compiled step-kernel shape: lanes per object, lane-group pairs, thread bound
template <int L_, bool PAIR_, int MAXT_>
struct Shape {
    static constexpr int L = L_;
    static constexpr bool PAIR = PAIR_;
    static constexpr int MAXT = MAXT_;
};

// The instantiated shapes: 1, 2, 4, 8, 16 lanes at the wide thread bound;
// pairs at 1, 2, 4 lanes (slower at 8 and 16); the deep bound at 2 and 4
// lanes, paired or not.  Anything else returns `bad`.
template <class R, class F>
static R dispatch(int lanes, int pair, int deep, R bad, F&& f) {
    if (deep && hasDeepShape(lanes)) {
        if (lanes == 2) return pair ? f(Shape<2, true, kDeepThreads>{}) : f(Shape<2, false, kDeepThreads>{});
        return pair ? f(Shape<4, true, kDeepThreads>{}) : f(Shape<4, false, kDeepThreads>{});
    }
    if (deep) return bad;
    if (pair) {
        switch (lanes) {
            case 1: return f(Shape<1, true, maxStepThreads(1)>{});
            case 2: return f(Shape<2, true, maxStepThreads(2)>{});
            case 4: return f(Shape<4, true, maxStepThreads(4)>{});
            default: return bad;
        }
    }
    switch (lanes) {
        case 1: return f(Shape<1, false, maxStepThreads(1)>{});
        case 2: return f(Shape<2, false, maxStepThreads(2)>{});
        case 4: return f(Shape<4, false, maxStepThreads(4)>{});
        case 8: return f(Shape<8, false, maxStepThreads(8)>{});
        case 16: return f(Shape<16, false, maxStepThreads(16)>{});
        default: return bad;
    }
}

template <class S>
static auto kernelOf() {
    return propagateKernel<S::L, PHOP_T, (bool)PHOP_SG, S::PAIR, S::MAXT>;
}

cudaError_t PHOP_CAT(launchPropagate_, PHOP_SUFFIX)(const StepParams& p, size_t paramsBytes, int lanes, int ctas,
                                                    int threads, int smem, cudaStream_t stream) {
    if (paramsBytes != sizeof(StepParams)) return cudaErrorInvalidValue;  // objects built from different headers
    return dispatch(lanes, p.pairSh, p.deepRegs, cudaErrorInvalidValue, [&](auto shape) -> cudaError_t {
        auto k = kernelOf<decltype(shape)>();
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
        }
        k<<<ctas, threads, smem, stream>>>(p);
        return cudaGetLastError();
    });
}

int PHOP_CAT(occupancy_, PHOP_SUFFIX)(int lanes, int pair, int deep, int threads, int smem) {
    return dispatch(lanes, pair, deep, 0, [&](auto shape) -> int {
        auto k = kernelOf<decltype(shape)>();
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem);
        return n;
    });
}

cudaError_t PHOP_CAT(attributes_, PHOP_SUFFIX)(int lanes, int pair, int deep, cudaFuncAttributes* a) {
    return dispatch(lanes, pair, deep, cudaErrorInvalidValue, [&](auto shape) -> cudaError_t {
        return cudaFuncGetAttributes(a, kernelOf<decltype(shape)>());
    });
}

}  // namespace phop
