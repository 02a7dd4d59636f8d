// Fused batched RKF78 propagation kernels for sm_100a.
//
// One persistent kernel advances object groups through all their fixed steps:
// the 13 RKF78 stages, the full force model and the 8th-order update run on
// chip (registers and shared memory), so the only per-object HBM traffic is the
// state read at the start and written at the end of the whole propagation.
//
// Work split (autotuned):  L lanes (1, 2, 4, 8 or 16) cooperate on one object,
// a warp holds 32/L objects.
//   * RK state: lane j of a group owns the state components d with d % L == j,
//     keeps y_d in registers and the 13 stage derivatives k_s[d] in shared
//     memory ([stage][component][thread], conflict-free), forms the
//     stage state for its components in the reference's order
//     (parm/integrate/rk/host/Step.h:33-84) and the 8th-order update in stage
//     order (Step.h:86-104), and broadcasts components by warp shuffle.
//   * Spherical harmonics: orders m are processed in blocks of L columns, lane
//     j taking m = bL + j.  Every lane advances the diagonal P_mm, dP_mm,
//     cos/sin(m lambda) and alpha^m with the reference's recurrences
//     (LegendreRecursor.h:202-208, PseudoPhasor.h:58-64), so the column start
//     values are the reference's.  The n <= 8 part of each column (with the
//     epoch's tide deltas folded into n <= 6) is always FP64; the n > 8 part
//     runs in the tile type T (double, or float for split precision) from a
//     lane-interleaved coefficient tile that a TMA bulk copy stages into
//     shared memory, so the L lanes of a group read one contiguous line per
//     term and the groups of a warp share it by broadcast.  Per column the
//     sums  sum (n+1) c Pt, sum (n+1) s Pt, sum c dPt, sum s dPt, sum c Pt,
//     sum s Pt  (Pt = alpha^n P) are accumulated and the phasor applied once,
//     which is algebraically the reference's per-term phase product
//     (DegreeLoop.h:83-112).  Partial accelerations are folded across the
//     group by xor shuffles.
//   * Everything else (third bodies, SRP with shadow, NRLMSISE-00 drag,
//     relativity) is evaluated by every lane of the group on the broadcast
//     stage state.
//
// Time grid: batches whose objects share epoch, step and duration read the
// per-step start / step size and the per-stage EpochRecord from tables made
// before the launch; mixed batches keep per-object time (FixedStep.h:30-37
// per object) and form each stage's record by 4-point Lagrange interpolation
// in an epoch-record grid of at most 30 s spacing that spans the batch, with
// the NRLMSISE-00 time inputs (seconds of day, sidereal time, weather slot)
// evaluated exactly at the stage epoch.
#pragma once
#include <stdint.h>

#include "device_env.cuh"

namespace phop {

// Each column's low degrees run in FP64 from the LowTable (with the epoch's
// tide deltas for n <= 6); the tile holds the degrees above.  The FP64 form
// starts its tile at n = 9; split precision keeps n <= splitFp64Degree
// (by default 20, or 24 for fields above degree 80; at most kLowMax) in FP64
// and runs the rest in FP32.
constexpr int kLowDeg = 8;                                  // FP64 form: n <= 8 from the LowTable
constexpr int kSplitFp64Degree = 20;                        // split form default up to degree 80
constexpr int kSplitFp64DegreeHigh = 24;                    // split form default above degree 80
constexpr int kLowMax = 24;                                 // largest FP64 low part
constexpr int kLowTri = (kLowMax + 2) * (kLowMax + 3) / 2;  // factor triangle up to n = kLowMax + 1

// coefficient tile entry for the n > 8 part: c, s, (n+1)c, (n+1)s and the
// recursion factors a, b of the step n -> n+1
struct __align__(16) TileD {
    double c, s, cp, sp, a, b;
};
struct __align__(16) TileF {
    float c, s, cp, sp, a, b, pad0, pad1;
};
template <typename T> struct TileOf;
template <> struct TileOf<double> { using type = TileD; };
template <> struct TileOf<float> { using type = TileF; };

// low-degree FP64 table (n <= kLowMax coefficients, factors to n = kLowMax + 1)
struct LowTable {
    double C[kLowTri];
    double S[kLowTri];
    double a[kLowTri];
    double b[kLowTri];
};

struct StepParams {
    DevEnv env;
    int64_t n;          // objects
    double* state;      // SoA: x[n], y[n], z[n], vx[n], vy[n], vz[n]
    const double* bc;   // cd * area / mass  (km^2 / kg)
    const double* ams;  // cr * area / mass
    // shared time grid
    int nsteps;
    const double* stepT0;
    const double* stepDt;
    const EpochRecord* records;  // [nsteps][13]
    // trajectory records (uniform batches): after every trajEvery-th step the
    // states go to traj[r][component][object], object in input order
    double* traj;
    int trajEvery;
    int trajRecords;  // capacity of traj in records: writes beyond it are skipped
    // per-object time (mixed batches)
    double* cur;
    const double* end;
    double* dt;
    const double* step;
    int64_t maxSteps;
    int* unfinished;        // per object: 1 if it did not reach its end
    const int64_t* order;   // processing order of objects (nullable)
    // epoch-record grid of a mixed batch (nullable): grid[k] holds the record
    // at TDB seconds (gridBase + k) * gridH, k < gridN.  The grid is anchored
    // at multiples of gridH, so an object's interpolated records do not depend
    // on which other objects share its batch.
    const EpochRecord* grid;
    // the same grid as value pairs: gridPairs[k * kInterpFields + f] = field f
    // of records k and k + 1, so that a 4-point stencil reads each field with
    // two 16-byte loads from two records instead of four 8-byte loads
    const double2* gridPairs;
    double gridH;
    int64_t gridBase;
    int gridN;
    int64_t stride;  // SoA stride of `state` (0: n); object pools use their capacity
    // geopotential
    const void* tile;       // tile entries in global memory
    int tileBytes;          // multiple of 16
    const int2* blocks;     // per block: entry offset, length
    int nblocks;
    const LowTable* low;
    const double* diagC;    // c_m, m = 0..M
    const double2* diagStep;  // per m: (c_{m+1}...c_{m+L}, same x (m+L)/m), nullable
    int lowDeg;             // n <= lowDeg of every column in FP64 from `low`; the tile starts at lowDeg + 1
    const void* tile64;     // split precision: the FP64 tile (global memory, same blocks)
    double splitRadius;     // split precision: radius (km) below which the tile part stays FP64; 0 = none
    int useSmemTile;
    int pairSh;             // the geopotential of lane-group pairs (tile built for 2L lanes)
    int deepRegs;           // host-side choice of the kernel's thread bound (stepThreadBound)
    int tileWaitTest;       // test of the staging time-out: arm the barrier, issue no copy
    // scheduling and errors
    int* workCounter;
    int* errorFlag;
    int* tileFallbacks;     // CTAs whose tile staging timed out (read the tile from global memory); nullable
};

// Threads per CTA the step kernel is compiled for: narrow lane splits run one
// CTA of few threads per SM (the coefficient tile fills shared memory), so
// they get up to 255 registers per thread instead of spilling at 128.  The
// "wide" shape below, and at two and four lanes also a "deep" one of
// kDeepThreads threads: 255 registers a thread instead of 168 (fewer warps,
// fewer spills; the autotuner times both).
__host__ __device__ constexpr int maxStepThreads(int lanes) {
    return lanes == 1 ? 256 : lanes == 2 ? 320 : 384;
}
constexpr int kDeepThreads = 256;
__host__ __device__ constexpr bool hasDeepShape(int lanes) { return lanes == 2 || lanes == 4; }
__host__ __device__ constexpr int stepThreadBound(int lanes, int deep) {
    return deep && hasDeepShape(lanes) ? kDeepThreads : maxStepThreads(lanes);
}

void launchEpochRecords(const DevEnv& env, const double* epochs, int count, EpochRecord* out, cudaStream_t stream);
// pairs[(k * kInterpFields + f)] = {field f of grid[k], of grid[k + 1]}, k < count - 1
void launchRecordPairs(const EpochRecord* grid, int64_t count, double2* pairs, cudaStream_t stream);
cudaError_t launchPropagate(const StepParams& p, int lanes, bool split, bool shared, int ctas, int threads,
                            cudaStream_t stream);
int propagateSmemBytes(const StepParams& p, int lanes, int threads);
int propagateMaxCtasPerSm(int lanes, bool split, bool shared, int pair, int deep, int threads, int smem);
// The compiled instantiation's attributes (maxThreadsPerBlock, numRegs,
// localSizeBytes): the launch shape never asks for more threads than the
// instantiation accepts.
cudaError_t propagateAttributes(int lanes, bool split, bool shared, int pair, int deep, cudaFuncAttributes* a);

}  // namespace phop
