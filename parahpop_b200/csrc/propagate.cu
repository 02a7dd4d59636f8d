// Epoch-record kernel and launch dispatch for the fused propagation kernels
// (kernel bodies: propagate_impl.cuh; instantiations: propagate_inst.cu).
#include <cuda_runtime.h>

#include "propagate.cuh"

namespace phop {

#define PHOP_DECL(sfx)                                                                                     \
    cudaError_t launchPropagate_##sfx(const StepParams& p, size_t paramsBytes, int lanes, int ctas, int threads, \
                                      int smem, cudaStream_t stream);                                       \
    int occupancy_##sfx(int lanes, int threads, int smem);
PHOP_DECL(f64_grid)
PHOP_DECL(f64_mixed)
PHOP_DECL(f32_grid)
PHOP_DECL(f32_mixed)
#undef PHOP_DECL

__global__ void epochRecordsKernel(const __grid_constant__ DevEnv env, const double* __restrict__ epochs, int count,
                                   EpochRecord* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    EpochRecord r;
    evalEpochRecord(env, epochs[i], r);
    out[i] = r;
}

void launchEpochRecords(const DevEnv& env, const double* epochs, int count, EpochRecord* out, cudaStream_t stream) {
    if (count <= 0) return;
    const int threads = 64;
    epochRecordsKernel<<<(count + threads - 1) / threads, threads, 0, stream>>>(env, epochs, count, out);
}

int propagateSmemBytes(const StepParams& p, int lanes, int threads) {
    const int cpl = (6 + lanes - 1) / lanes;
    return (p.useSmemTile ? p.tileBytes : 0) + 13 * cpl * threads * (int)sizeof(double);
}

int propagateMaxCtasPerSm(int lanes, bool split, bool shared, int threads, int smem) {
    if (split) return shared ? occupancy_f32_grid(lanes, threads, smem) : occupancy_f32_mixed(lanes, threads, smem);
    return shared ? occupancy_f64_grid(lanes, threads, smem) : occupancy_f64_mixed(lanes, threads, smem);
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
