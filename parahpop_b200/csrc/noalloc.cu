// Propagation entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they propagate: a
// plug-in inside a host application whose own pool allocator has reserved
// the GPU's memory, a real-time loop that cannot afford the device-wide
// synchronisation a cudaMalloc or cudaFree may imply, or a service that
// fixes its memory footprint at start-up and must not grow it.  For them
// this entry point runs the same two kernels as phop_propagate_device (epoch
// records, then the fused step kernel) but takes every scratch buffer from
// one file-scope device array, kStaticScratchBytes large, carved as:
//
//   control words (work counter, error flag)     256 B
//   coefficient tile + block table               kTileBytes + kBlockBytes
//   step start / size tables                     2 x kMaxSteps doubles
//   stage epochs                                 13 x kMaxSteps doubles
//   epoch records                                13 x kMaxSteps records
//
// Limits: at most kMaxSteps (256) fixed steps per call and a coefficient tile
// of at most kTileBytes (512 KiB, enough for degree/order 120 in FP64); calls
// beyond them are rejected with an error.  Every GPU that loads the library
// holds the array (4 MiB) until the process exits.  All calls share it: the
// control words are cleared on every call, the tile is re-copied whenever a
// call needs another one than the array holds (keyed by the context's
// never-reused serial number, the lane count and the precision), and calls
// whose work overlaps on the GPU race on the array, so the caller must order
// them (one stream, or events).  The call is synchronous: it returns once
// the propagation has finished on the GPU and its error flag has been read.
// The first call on a device resolves the array's device address
// (cudaGetSymbolAddress); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "engine.hpp"

namespace phop {

constexpr size_t kStaticScratchBytes = 4u << 20;
constexpr int kMaxSteps = 256;
constexpr size_t kCtlBytes = 256;
constexpr size_t kTileBytes = 512u << 10;
constexpr size_t kBlockBytes = 4u << 10;

static __device__ __align__(256) unsigned char g_staticScratch[kStaticScratchBytes];

namespace {
struct DeviceScratch {
    unsigned char* base = nullptr;  // device address of g_staticScratch on this device
    uint64_t tileOwner = 0;         // serial number of the context whose tile the array holds (0: none)
    int tileKey = -1;
};
DeviceScratch g_scratch[64];
std::mutex g_scratchMutex;

static_assert(kCtlBytes + kTileBytes + kBlockBytes + 2 * kMaxSteps * sizeof(double) + 13 * kMaxSteps * sizeof(double)
                      + 13 * kMaxSteps * sizeof(EpochRecord) + 1024
                  <= kStaticScratchBytes,
              "static scratch layout does not fit");
}  // namespace

// Host copy of the lane-interleaved coefficient tile (same layout as the
// engine's device tiles, propagate.cuh), kept so the allocation-free entry
// point can copy it into the static array without allocating.
static double tileFactorA(int n, int m, bool norm) {
    const double nn = n, mm = m;
    return norm ? std::sqrt(((2.0 * nn - 1.0) * (2.0 * nn + 1.0)) / ((nn - mm) * (nn + mm))) : (2.0 * nn - 1.0) / (nn - mm);
}
static double tileFactorB(int n, int m, bool norm) {
    const double nn = n, mm = m;
    return norm ? std::sqrt(((2.0 * nn + 1.0) * (nn + mm - 1.0) * (nn - mm - 1.0)) / ((2.0 * nn - 3.0) * (nn + mm) * (nn - mm)))
                : (nn + mm - 1.0) / (nn - mm);
}

const Engine::HostTile& Engine::hostTileFor(int L, bool split, int lowDeg) {
    const int key = (lowDeg * 32 + L) * 2 + (split ? 1 : 0);
    auto it = hostTiles_.find(key);
    if (it != hostTiles_.end()) return it->second;
    const HostEnvironment& h = host_;
    const int N = h.shDegree, M = h.shOrder;
    const bool norm = h.shNormalized != 0;
    const int nb = h.hasShape ? (M + 1 + L - 1) / L : 0;
    HostTile out;
    out.nblocks = nb;
    out.blocks.assign(nb > 0 ? nb : 1, int2{0, 0});
    std::vector<TileD> entries;
    for (int b = 0; b < nb; ++b) {
        const int n0b = std::max(b * L, lowDeg + 1);
        const int len = std::max(0, N - n0b + 1);
        out.blocks[b] = int2{(int)entries.size(), len};
        const size_t base = entries.size();
        entries.resize(base + (size_t)len * L, TileD{0, 0, 0, 0, 0, 0});
        for (int j = 0; j < L; ++j) {
            const int m = b * L + j;
            if (m > M) continue;
            const int n0 = std::max(m, lowDeg + 1);
            for (int i = 0; i < len; ++i) {
                const int n = n0 + i;
                if (n > N) break;
                TileD& t = entries[base + (size_t)i * L + j];
                const size_t ti = (size_t)n * (n + 1) / 2 + m;
                t.c = h.shC[ti];
                t.s = m > 0 ? h.shS[ti] : 0.0;
                t.cp = (double)(n + 1) * t.c;
                t.sp = (double)(n + 1) * t.s;
                if (n + 1 <= N) {
                    t.a = tileFactorA(n + 1, m, norm);
                    t.b = tileFactorB(n + 1, m, norm);
                }
            }
        }
    }
    if (split) {
        std::vector<TileF> f(entries.size());
        for (size_t k = 0; k < entries.size(); ++k)
            f[k] = TileF{(float)entries[k].c, (float)entries[k].s, (float)entries[k].cp, (float)entries[k].sp,
                         (float)entries[k].a, (float)entries[k].b, 0.f, 0.f};
        out.bytes.resize(f.size() * sizeof(TileF));
        std::memcpy(out.bytes.data(), f.data(), out.bytes.size());
    } else {
        out.bytes.resize(entries.size() * sizeof(TileD));
        std::memcpy(out.bytes.data(), entries.data(), out.bytes.size());
    }
    out.bytes.resize((out.bytes.size() + 15) / 16 * 16 + 16, 0);
    return hostTiles_.emplace(key, std::move(out)).first->second;
}

// Device address of the static scratch array on `device` (set up once per
// device, with that device current).
static DeviceScratch& scratchFor(int device) {
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (device < 0 || device >= 64) throw std::runtime_error("device index out of range");
    DeviceScratch& s = g_scratch[device];
    if (!s.base) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_staticScratch);
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("cudaGetSymbolAddress of the static scratch failed: ")
                                     + cudaGetErrorString(e));
        s.base = (unsigned char*)ptr;
    }
    return s;
}

void Engine::propagateNoAlloc(int64_t n, double* dState, const double* dBc, const double* dAms, double epochMjd,
                              double duration, double step, int64_t maxSteps, const RunOptions& opt,
                              double* outEpochMjd, cudaStream_t stream) {
    if (cudaSetDevice(device_) != cudaSuccess) throw std::runtime_error("cannot select the context's device");
    if (opt.lanes != 0 && opt.lanes != 1 && opt.lanes != 2 && opt.lanes != 4 && opt.lanes != 8 && opt.lanes != 16)
        throw std::runtime_error("lanes must be 1, 2, 4, 8 or 16");
    if (opt.split && opt.splitFloorKm > 0.0)
        throw std::runtime_error("the allocation-free entry point does not take the split_floor_km option "
                                 "(it would need the FP64 tile beside the FP32 one)");
    DeviceScratch& ds = scratchFor(device_);
    // shared time grid (FixedStep.h:7-37)
    const double start = std::fma(epochMjd, 86400.0, -43200.0);
    const double end = std::fma(epochMjd + duration / 86400.0, 86400.0, -43200.0);
    const double span = end - start;
    if (!(span > 0) || !std::isfinite(span))
        throw std::runtime_error("Duration/step cannot be represented by the integration time/index types.");
    double t0[kMaxSteps], dtv[kMaxSteps], stageT[13 * kMaxSteps];
    double cur = start, d = std::min(step, span);
    int K = 0;
    bool done = false;
    while (!done) {
        if (K >= maxSteps) throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
        if (K >= kMaxSteps)
            throw std::runtime_error("the allocation-free entry point takes at most " + std::to_string(kMaxSteps)
                                     + " steps per call");
        t0[K] = cur;
        dtv[K] = d;
        ++K;
        cur += d;
        const double rem = end - cur;
        done = rem <= 0;
        d = done ? 0 : std::min(step, rem);
    }
    static const double c[12] = {2. / 27, 1. / 9, 1. / 6, 5. / 12, 1. / 2, 5. / 6, 1. / 6, 2. / 3, 1. / 3, 1.0, 0, 1.0};
    for (int k = 0; k < K; ++k)
        for (int s = 0; s < 13; ++s) stageT[k * 13 + s] = s == 0 ? t0[k] : std::fma(dtv[k], c[s - 1], t0[k]);
    // carve the static array
    unsigned char* p = ds.base;
    int* ctl = (int*)p;
    p += kCtlBytes;
    void* tileDst = p;
    p += kTileBytes;
    int2* blocksDst = (int2*)p;
    p += kBlockBytes;
    double* dT0 = (double*)p;
    p += kMaxSteps * sizeof(double);
    double* dDt = (double*)p;
    p += kMaxSteps * sizeof(double);
    double* dStage = (double*)p;
    p += 13 * kMaxSteps * sizeof(double);
    EpochRecord* dRec = (EpochRecord*)p;
    // coefficient tile (host copy kept by the engine) into the array
    const int L = opt.lanes > 0 ? opt.lanes : autoLanes(n);
    const int lowDeg = lowDegreeFor(opt, host_.shDegree);
    const HostTile& ht = hostTileFor(L, opt.split, lowDeg);
    if (ht.bytes.size() > kTileBytes || ht.blocks.size() * sizeof(int2) > kBlockBytes)
        throw std::runtime_error("coefficient tile exceeds the allocation-free entry point's 512 KiB limit");
    const int key = (lowDeg * 32 + L) * 2 + (opt.split ? 1 : 0);
    auto check = [](cudaError_t e) {
        if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    };
    {
        // the array's tile belongs to the last call's (context, lanes,
        // precision); a context's serial number is never reused, so a new
        // context at a freed one's address still gets its own tile
        std::lock_guard<std::mutex> lock(g_scratchMutex);
        if (ds.tileOwner != serial_ || ds.tileKey != key) {
            ds.tileOwner = 0;
            check(cudaMemcpyAsync(tileDst, ht.bytes.data(), ht.bytes.size(), cudaMemcpyHostToDevice, stream));
            check(cudaMemcpyAsync(blocksDst, ht.blocks.data(), ht.blocks.size() * sizeof(int2),
                                  cudaMemcpyHostToDevice, stream));
            ds.tileOwner = serial_;
            ds.tileKey = key;
        }
    }
    check(cudaMemcpyAsync(dT0, t0, K * sizeof(double), cudaMemcpyHostToDevice, stream));
    check(cudaMemcpyAsync(dDt, dtv, K * sizeof(double), cudaMemcpyHostToDevice, stream));
    check(cudaMemcpyAsync(dStage, stageT, 13 * K * sizeof(double), cudaMemcpyHostToDevice, stream));
    check(cudaMemsetAsync(ctl, 0, kCtlBytes, stream));
    launchEpochRecords(denv_, dStage, 13 * K, dRec, stream);
    check(cudaGetLastError());
    StepParams sp{};
    sp.env = denv_;
    sp.n = n;
    sp.state = dState;
    sp.bc = dBc;
    sp.ams = dAms;
    sp.nsteps = K;
    sp.stepT0 = dT0;
    sp.stepDt = dDt;
    sp.records = dRec;
    sp.maxSteps = maxSteps;
    sp.tile = tileDst;
    sp.tileBytes = (int)ht.bytes.size();
    sp.blocks = blocksDst;
    sp.nblocks = ht.nblocks;
    sp.low = dLow_;
    sp.lowDeg = lowDeg;
    sp.diagC = dDiag_;
    sp.workCounter = ctl;
    sp.errorFlag = ctl + 1;
    const int threadsReq = std::min(opt.threads > 0 ? opt.threads : 512, maxStepThreads(L));
    const int kPerThread = 13 * ((6 + L - 1) / L) * 8;
    int threads;
    if (opt.tileSmem != 0 && (int)ht.bytes.size() + 1024 + 64 * kPerThread <= maxSmem_) {
        sp.useSmemTile = 1;
        threads = std::min(threadsReq, (maxSmem_ - (int)ht.bytes.size() - 1024) / kPerThread / 32 * 32);
    } else {
        sp.useSmemTile = 0;
        threads = std::min(threadsReq, (maxSmem_ - 1024) / kPerThread / 32 * 32);
    }
    const int smem = propagateSmemBytes(sp, L, threads);
    int perSm = opt.ctasPerSm > 0 ? opt.ctasPerSm : propagateMaxCtasPerSm(L, opt.split, true, 0, 0, threads, smem);
    if (perSm <= 0) perSm = 1;
    const int64_t groups = (n + (32 / L) - 1) / (32 / L);
    const int64_t need = (groups + threads / 32 - 1) / (threads / 32);
    const int ctas = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms_ * perSm, need));
    check(launchPropagate(sp, L, opt.split, true, ctas, threads, stream));
    int err = 0;
    check(cudaMemcpyAsync(&err, ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
    check(cudaStreamSynchronize(stream));
    if (err) throw std::runtime_error("Propagation kernel reported error " + std::to_string(err) + ".");
    if (outEpochMjd) *outEpochMjd = std::fma(cur, 1.0 / 86400.0, 0.5);
}

}  // namespace phop
