// Host engine: loads a ParaHPOP model configuration and its environment files,
// keeps the environment resident on one GPU and propagates batches of objects
// through the fused kernels.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "device_env.cuh"
#include "propagate.cuh"
#include "value.hpp"

namespace phop {

// spacing of the epoch-record grid of mixed batches (TDB seconds)
constexpr double kRecordGridSeconds = 30.0;

struct EphUnitHost {
    int target, center, nint, pdeg;
    double startEpoch, finalEpoch;
    std::vector<double> data;
};

// Everything read from the environment files, in host memory.
struct HostEnvironment {
    // constants
    double au = 0.0;
    std::map<int, double> constGm, constRadius, constJ2, constSoi;
    // bodies sorted by NAIF id
    struct Body {
        std::string name;
        int id = 0;
        int flags = 0;
        double gm = 0.0, radius = 0.0;
        double j2 = 0.0, gmConst = 0.0, soi = 1e20;  // oblateness model (constants file)
        double flattening = 0.0;                     // the body's "flattening" (geodetic height for drag)
    };
    std::vector<Body> bodies;
    double flattening = 0.0;
    // geopotential
    bool hasShape = false;
    int shDegree = 0, shOrder = 0, shNormalized = 1;
    double shR = 0.0, shGM = 0.0;
    std::vector<double> shC, shS;  // triangle n(n+1)/2+m, n <= shDegree
    // ephemeris
    std::vector<EphUnitHost> eph;
    // orientation (IERS2000 unit)
    bool hasRot = false;
    // the Earth frame in use: 4 = IERS2000 model unit (target 3001), 3 =
    // binary Chebyshev Euler angles (ITRF93, target 3000)
    int rotKind = 0;
    int rotNnut = 0, rotNerp = 0;      // kind 4: Lagrange node counts
    int rotNint = 0, rotPdeg = 0;      // kind 3: Chebyshev intervals and degree
    int rotEcliptic = 0;               // kind 3: angles relative to ECLIPJ2000 (inertialFrame 17)
    // kind 1 (IAU body model, degrees): coefficient counts of the RA, Dec
    // and PM polynomials and of their nutation-precession amplitudes; the
    // barycentric angle polynomials follow the body data in rotData at
    // iauBaryOffset (-1: none), iauNpAngles of iauNpDeg coefficients each
    int iauDeg[3] = {0, 0, 0}, iauNp[3] = {0, 0, 0};
    int iauBaryOffset = -1, iauNpDeg = 0, iauNpAngles = 0;
    double rotStart = 0.0, rotFinal = 0.0;
    std::vector<double> rotData;
    std::string earthOrientation;      // bodies.Earth.orientation (empty: the unique loaded frame)
    // exponential atmosphere bands {rho0, h0, scaleHeight, hCutoff}, ascending h0
    std::vector<std::array<double, 4>> expSeg;
    // NRLMSISE-00
    bool hasNrl = false;
    double nrlStartMjd = 0.0, nrlHcutoff = 1000.0, nrlDensityScale = 1.0;
    std::vector<double> nrlWeather;  // 13 x ndays
    int nrlNdays = 0;
    // Earth corrections
    bool solid = false, ocean = false, relativity = false, zeroTide = true;
    double eopFirstMjd = 0.0;
    std::vector<double> eop;  // 4 x n
    int eopN = 0;
    // bodies other than the Earth with the J2 model, each with its IAU body
    // model (coefficients, then its barycentric angle polynomials)
    struct PoleBody {
        int bodyIndex = -1;
        int deg[3] = {0, 0, 0}, np[3] = {0, 0, 0};
        int baryOffset = -1, npDeg = 0;
        std::vector<double> data;
    };
    std::vector<PoleBody> poles;
    // the body whose field the geopotential is (one per configuration) and,
    // for a body other than the Earth, its IAU body model
    int shBodyId = 399;
    PoleBody shFrame;
    // the body whose atmosphere the exponential model describes (one per configuration)
    int atmBodyId = 399;
};

// Loads the environment of a `model` configuration object (the reference's
// interface::config::Model input); relative paths must already be resolved.
void loadEnvironment(const Value& model, HostEnvironment& env);

// 64-bit FNV-1a digest of every loaded field, for comparing loads.
uint64_t environmentDigest(const HostEnvironment& env);

// Per-object inputs in the reference's target schema (driver.cpp:97-123).
struct TargetSet {
    std::vector<int64_t> ids;
    std::vector<double> epoch;     // MJD2000 TDB
    std::vector<double> state;     // n x 6, km and km/s
    std::vector<double> mass, dragArea, srpArea, cd, cr;
    std::vector<double> duration;  // s, per object
    std::vector<double> step;      // s, per object
    size_t size() const { return ids.size(); }
};

struct RunStats {
    double kernelMs = 0.0;         // step kernel, CUDA events
    double recordsMs = 0.0;        // epoch-record kernel
    double tuneMs = 0.0;           // lane-count autotuner probes (first batch of a size class)
    double totalMs = 0.0;          // whole propagate call incl. copies
    int64_t objectSteps = 0;       // sum over objects of steps taken
    int64_t launches = 0;          // kernels launched by this call
    int lanes = 0;
    int ctas = 0;
    int threads = 0;
    bool split = false;
    bool sharedGrid = false;
    bool tileInSmem = false;
    bool pairSh = false;           // the geopotential of lane-group pairs was used
    bool deepRegs = false;         // the deep thread bound (256 threads, 255 registers) was used
    int registers = 0;             // registers a thread of the step kernel used
    int64_t tileFallbacks = 0;     // CTAs that read the tile from global memory after a staging time-out
};

struct RunOptions {
    int lanes = 0;     // 0: autotuned
    int threads = 512;
    bool split = false;
    int ctasPerSm = 0; // 0: occupancy
    bool ordered = true;  // process objects in order of geocentric radius
    bool graph = true;    // launch the step as a cached CUDA graph
    double splitFloorKm = 0.0;  // split precision: FP64 tile part below this height over the field radius
    int splitFp64Degree = 0;  // split precision: degrees n <= this stay FP64 (8 .. kLowMax); 0 = by field degree
    int tileSmem = -1;    // coefficient tile in shared memory: -1 when it fits, 0 never (read through L1)
    int mixedOrder = 0;   // mixed batches inside a step-count bucket: 0 radius, 1 epoch, 2 drag band + epoch
    int tileWaitTest = 0; // test of the tile-staging time-out: the barrier is armed, no copy issued
    int pairSh = -1;      // geopotential of lane-group pairs (packed FP32 in split precision): 1 on, 0 off,
                          // -1 autotuned with the lane count (pinned lanes: on up to 4 lanes)
    int deepRegs = -1;    // thread bound at 2 and 4 lanes: 1 deep (256 threads, 255 registers), 0 wide
                          // (320 / 384 threads, 168 registers), -1 autotuned (pinned lanes: wide)
    // trajectory records of a uniform batch: device buffer of
    // (steps / trajEvery) x 6 x n doubles, null for none
    double* dTraj = nullptr;
    int trajEvery = 0;
    int trajRecords = 0;  // capacity of dTraj in records
};

// degrees n <= this of every column run in FP64 from the LowTable
int lowDegreeFor(const RunOptions& opt, int fieldDegree);

class Engine {
public:
    Engine(const HostEnvironment& env, int device);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    const HostEnvironment& environment() const { return host_; }

    // Checks that ephemeris / orientation / EOP data cover [loMjd, hiMjd].
    void assertCoverage(double loMjd, double hiMjd) const;

    // Propagates `t` in place: final MJD2000 epochs and states (n x 6).
    // Per-object duration / step.  Throws on error.
    void propagate(const TargetSet& t, int64_t maxSteps, const RunOptions& opt, std::vector<double>& outEpoch,
                   std::vector<double>& outState, RunStats* stats, cudaStream_t stream = 0);

    // Device-resident variant: `state` is an SoA device array (6 x n) updated in
    // place; other inputs are host arrays.  Used for timing with inputs held
    // in HBM.
    void propagateResident(int64_t n, double* dState, const double* epochMjd, const double* bc, const double* ams,
                           double duration, double step, int64_t maxSteps, const RunOptions& opt,
                           std::vector<double>& outEpochMjd, RunStats* stats, cudaStream_t stream = 0);

    // Sliced per-object-time batch resident in device memory: dTime holds
    // cur[n], end[n], dt[n], step[n] (TDB seconds past J2000; dt = 0 once an
    // object has reached its end), updated in place; every unfinished
    // object advances by at most maxSteps fixed steps.  Returns the number
    // of objects still short of their end.
    int64_t advanceObjects(int64_t n, double* dState, double* dTime, const double* dBc, const double* dAms,
                           int64_t maxSteps, const RunOptions& opt, RunStats* stats, cudaStream_t stream = 0);

    int device() const { return device_; }
    int smCount() const { return sms_; }
    int autoLanes(int64_t n) const;

    // Allocation-free variant of propagateResident (noalloc.cu): scratch comes
    // from a file-scope device array; dBc / dAms are device arrays.
    void propagateNoAlloc(int64_t n, double* dState, const double* dBc, const double* dAms, double epochMjd,
                          double duration, double step, int64_t maxSteps, const RunOptions& opt,
                          double* outEpochMjd, cudaStream_t stream = 0);

    // internal
    struct HostTile {
        std::vector<unsigned char> bytes;
        std::vector<int2> blocks;
        int nblocks = 0;
    };
    struct Tile {
        void* dTile = nullptr;
        int2* dBlocks = nullptr;
        double2* dDiagStep = nullptr;
        int bytes = 0;
        int nblocks = 0;
    };

    // Launch geometry of one step-kernel launch.
    struct LaunchShape {
        int lanes = 0, threads = 0, ctas = 0;
        int registers = 0;  // registers a thread of the chosen instantiation
        bool smemTile = false;
    };
    // Per-batch time description handed to the step kernel.
    struct TimeGrid {
        bool shared = false;
        // shared grid: per-step start epochs and sizes
        std::vector<double> t0, dt;
        // per-object time (device arrays) and the batch's record grid
        double *cur = nullptr, *end = nullptr, *dt1 = nullptr, *step = nullptr;
        int* unfinished = nullptr;
        const EpochRecord* grid = nullptr;
        const double2* gridPairs = nullptr;
        double gridH = 0.0;
        int64_t gridBase = 0;
        int gridN = 0;
        int64_t stride = 0;  // SoA stride of the state (0: n)
    };

private:
    friend class Server;
    const Tile& tileFor(int lanes, bool split, int lowDeg);
    const HostTile& hostTileFor(int lanes, bool split, int lowDeg);
    void uploadEnvironment();
    void* scratch(const std::string& name, size_t bytes);
    // device order of objects by increasing geocentric radius (SoA state of
    // stride `stride`); `slots` (nullable) lists the objects to order
    const int64_t* orderByRadius(int64_t n, const double* dState, cudaStream_t stream, int64_t* launches,
                                 int64_t stride = 0, const int64_t* slots = nullptr);
    void buildRecordGrid(double lo, double hi, TimeGrid& g, cudaStream_t stream, int64_t* launches);
    LaunchShape launchStep(StepParams p, int lanes, const RunOptions& opt, bool shared, cudaStream_t stream);
    LaunchShape prepareStep(StepParams& p, int lanes, const RunOptions& opt, bool shared);
    void enqueueStep(const StepParams& p, const LaunchShape& shape, const RunOptions& opt, bool shared,
                     cudaStream_t stream);
    void launchStepGraph(const StepParams& p, const LaunchShape& shape, const RunOptions& opt, bool shared,
                         cudaStream_t stream);
    struct GraphEntry {
        unsigned char params[sizeof(StepParams)];
        int lanes = 0, threads = 0, ctas = 0, flags = 0;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<GraphEntry> graphs_;
    // epoch records of the per-object-time path at grid indices [gridKLo_, gridKHi_]
    EpochRecord* gridCache_ = nullptr;
    double2* pairCache_ = nullptr;  // gridCache_ as value pairs (StepParams::gridPairs)
    int64_t gridKLo_ = 0, gridKHi_ = -1;
    cudaStream_t captureStream_ = nullptr;
    // autotuned launch shape of a batch class: lanes * 2 + (pairs ? 1 : 0)
    int tunedShape(const StepParams& base, const RunOptions& opt, bool shared, cudaStream_t stream, int64_t* launches);
    void runKernel(int64_t n, double* dState, const double* dBc, const double* dAms, const TimeGrid& g,
                   const int64_t* dOrder, int64_t maxSteps, const RunOptions& opt, RunStats* stats,
                   cudaStream_t stream, int64_t launchesBefore);

    HostEnvironment host_;
    uint64_t serial_ = 0;  // unique per context in this process, never reused (1, 2, ...)
    int device_ = 0;
    int sms_ = 0;
    int maxSmem_ = 0;
    DevEnv denv_{};
    std::vector<void*> owned_;
    std::map<std::string, std::pair<void*, size_t>> scratch_;
    std::map<int, Tile> tiles_;
    std::map<int, HostTile> hostTiles_;
    LowTable* dLow_ = nullptr;
    double* dDiag_ = nullptr;
    std::map<int, int> tuned_;  // autotuned lane count per batch class
    std::map<int64_t, int> occupancy_;  // resident CTAs per SM by launch configuration
    std::map<int, std::pair<int, int>> attrs_;  // maxThreadsPerBlock, numRegs of each step-kernel instantiation
};

}  // namespace phop
