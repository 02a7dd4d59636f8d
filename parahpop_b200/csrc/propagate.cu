// Epoch-record kernel and launch dispatch for the fused propagation kernels
// (kernel bodies: propagate_impl.cuh; instantiations: propagate_inst.cu).
#include <cuda_runtime.h>

#include "propagate.cuh"

namespace phop {

#define PHOP_DECL(sfx)                                                                                     \
    cudaError_t launchPropagate_##sfx(const StepParams& p, size_t paramsBytes, int lanes, int ctas, int threads, \
                                      int smem, cudaStream_t stream);                                       \
    int occupancy_##sfx(int lanes, int pair, int deep, int threads, int smem);                            \
    cudaError_t attributes_##sfx(int lanes, int pair, int deep, cudaFuncAttributes* a);
PHOP_DECL(f64_grid)
PHOP_DECL(f64_mixed)
PHOP_DECL(f32_grid)
PHOP_DECL(f32_mixed)
#undef PHOP_DECL

// One epoch record per thread; then the warp forms the tide corrections of
// its records one after the other, the terms split across its lanes
// (tidefield::tideDeltasWarp: lane s < 25 owns coefficient slot s).
__global__ void __launch_bounds__(64) epochRecordsKernel(const __grid_constant__ DevEnv env,
                                                         const double* __restrict__ epochs, int count,
                                                         EpochRecord* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < count;
    tidefield::Epoch tin;
    bool tides = false;
    if (live) {
        EpochRecord r;
        tides = evalEpochRecordBase(env, epochs[i], r, tin);
        out[i] = r;
    }
    if (!(env.solid || env.ocean)) return;
    __syncwarp();
    const int lane = threadIdx.x & 31;
    const int warpFirst = i - lane;
    unsigned todo = __ballot_sync(0xffffffffu, tides);
    while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        tidefield::Epoch ep;
        for (int k = 0; k < 9; ++k) ep.E[k] = __shfl_sync(0xffffffffu, tin.E[k], src);
        for (int k = 0; k < 3; ++k) {
            ep.sun[k] = __shfl_sync(0xffffffffu, tin.sun[k], src);
            ep.moon[k] = __shfl_sync(0xffffffffu, tin.moon[k], src);
        }
        ep.mjdUtc = __shfl_sync(0xffffffffu, tin.mjdUtc, src);
        ep.ut1Utc = __shfl_sync(0xffffffffu, tin.ut1Utc, src);
        ep.ttUtc = __shfl_sync(0xffffffffu, tin.ttUtc, src);
        ep.xp = __shfl_sync(0xffffffffu, tin.xp, src);
        ep.yp = __shfl_sync(0xffffffffu, tin.yp, src);
        double dC, dS;
        tidefield::tideDeltasWarp(ep, env.solid != 0, env.ocean != 0, env.zeroTide != 0, env.tideOcean,
                                  env.tideScale, dC, dS);
        if (lane < tidefield::kSlots) {
            out[warpFirst + src].dC[lane + 3] = dC;
            out[warpFirst + src].dS[lane + 3] = dS;
        }
    }
}

void launchEpochRecords(const DevEnv& env, const double* epochs, int count, EpochRecord* out, cudaStream_t stream) {
    if (count <= 0) return;
    const int threads = 64;
    epochRecordsKernel<<<(count + threads - 1) / threads, threads, 0, stream>>>(env, epochs, count, out);
}

static __global__ void recordPairsKernel(const EpochRecord* __restrict__ grid, int64_t total, double2* __restrict__ pairs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int64_t k = i / kInterpFields;
    const int f = (int)(i - k * kInterpFields);
    const double* a = (const double*)(grid + k);
    const double* b = (const double*)(grid + k + 1);
    pairs[i] = make_double2(a[f], b[f]);
}

void launchRecordPairs(const EpochRecord* grid, int64_t count, double2* pairs, cudaStream_t stream) {
    if (count < 2) return;
    const int64_t total = (count - 1) * kInterpFields;
    const int threads = 256;
    recordPairsKernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, stream>>>(grid, total, pairs);
}

int propagateSmemBytes(const StepParams& p, int lanes, int threads) {
    const int cpl = (6 + lanes - 1) / lanes;
    return (p.useSmemTile ? p.tileBytes : 0) + 13 * cpl * threads * (int)sizeof(double);
}

int propagateMaxCtasPerSm(int lanes, bool split, bool shared, int pair, int deep, int threads, int smem) {
    if (split)
        return shared ? occupancy_f32_grid(lanes, pair, deep, threads, smem)
                      : occupancy_f32_mixed(lanes, pair, deep, threads, smem);
    return shared ? occupancy_f64_grid(lanes, pair, deep, threads, smem)
                  : occupancy_f64_mixed(lanes, pair, deep, threads, smem);
}

cudaError_t propagateAttributes(int lanes, bool split, bool shared, int pair, int deep, cudaFuncAttributes* a) {
    if (split) return shared ? attributes_f32_grid(lanes, pair, deep, a) : attributes_f32_mixed(lanes, pair, deep, a);
    return shared ? attributes_f64_grid(lanes, pair, deep, a) : attributes_f64_mixed(lanes, pair, deep, a);
}

cudaError_t launchPropagate(const StepParams& p, int lanes, bool split, bool shared, int ctas, int threads,
                            cudaStream_t stream) {
    // every family checks the parameter block's size against its own view
    // of the layout (the families are separate translation units)
    const int smem = propagateSmemBytes(p, lanes, threads);
    const size_t b = sizeof(StepParams);
    if (split)
        return shared ? launchPropagate_f32_grid(p, b, lanes, ctas, threads, smem, stream)
                      : launchPropagate_f32_mixed(p, b, lanes, ctas, threads, smem, stream);
    return shared ? launchPropagate_f64_grid(p, b, lanes, ctas, threads, smem, stream)
                  : launchPropagate_f64_mixed(p, b, lanes, ctas, threads, smem, stream);
}

}  // namespace phop
