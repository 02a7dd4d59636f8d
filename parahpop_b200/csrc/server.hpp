// Serving loop: continuous batching of propagation requests on one GPU.
//
// Requests (batches of objects with their own epochs, durations and steps)
// are queued, admitted into a device-resident object pool while it has room
// (the pool's capacity is the HBM admission budget, fixed at creation) and
// while the running batch is within the compute budget (the objects one step
// of the measured rate covers in a slice, at least 65,536), and
// advanced together: every scheduling round launches the per-object-time step
// kernel once over all unfinished objects of all admitted requests, for as
// many fixed steps as fit a target time slice.  Requests that finish are
// copied out and their slots freed for the queue, so new requests join the
// running batch between slices instead of waiting for it to drain.
//
// An object's results do not depend on which requests share its slices: the
// lane split is fixed for the server's lifetime, epoch records come from a
// grid anchored at absolute epochs, and objects never interact.  The
// reference has no serving loop (its driver propagates one batch per process);
// this is the batching layer in front of the same propagation.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "engine.hpp"

namespace phop {

class Server {
public:
    enum State { Queued = 0, Running = 1, Done = 2, Failed = 3 };

    // capacity: objects resident at once (each slot holds 132 bytes of HBM);
    // sliceMs: target duration of one launch; maxSteps: per-request step cap
    // (the configuration's maxNumSteps).
    Server(Engine& engine, const RunOptions& opt, int64_t capacity, double sliceMs, int64_t maxSteps);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Queues a request; validated inputs as for Engine::propagate.
    int64_t submit(const TargetSet& t);
    // One scheduling round: admit, launch one slice, retire finished requests.
    // Returns the number of requests that finished (or failed) in this round.
    int step();
    State status(int64_t id) const;
    // Copies a finished request's results (epochs n, states n x 6) and forgets
    // it; throws the request's error if it failed.
    void take(int64_t id, double* outEpoch, double* outStates, double* latencyMs, double* queueMs);

    struct Stats {
        int64_t queued = 0, running = 0;
        int64_t done = 0, failed = 0;  // requests finished / failed since creation
        int64_t activeObjects = 0;
        int64_t launches = 0;          // kernels launched by the server
        int64_t rounds = 0;
        int64_t objectSteps = 0;       // object-steps of finished requests
        double busyMs = 0.0;           // step-kernel time (CUDA events)
        int lanes = 0;
    };
    Stats stats() const;

private:
    struct Request {
        int64_t id = 0;
        TargetSet t;
        State state = Queued;
        int64_t off = -1;              // first pool slot
        int64_t steps = 0;             // steps granted so far (per object)
        int64_t objectSteps = 0;       // sum of per-object step counts
        double lo = 0.0, hi = 0.0;     // TDB seconds spanned
        std::chrono::steady_clock::time_point submitted, admitted, finished;
        std::vector<double> outEpoch, outState;
        std::string error;
    };

    bool allocate(int64_t n, int64_t& off);
    void release(int64_t off, int64_t n);
    void admit(Request& r);
    void finish(Request& r);
    void ensureGrid(double lo, double hi);

    Engine& engine_;
    RunOptions opt_;
    int64_t capacity_;
    double sliceMs_;
    int64_t maxSteps_;
    int lanes_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    // pool (device), SoA with stride capacity_
    double *state_ = nullptr, *bc_ = nullptr, *ams_ = nullptr;
    double *cur_ = nullptr, *end_ = nullptr, *dt_ = nullptr, *step_ = nullptr;
    int* unfinished_ = nullptr;
    int64_t* active_ = nullptr;
    int* ctl_ = nullptr;
    std::vector<int> hostUnfinished_;
    std::map<int64_t, int64_t> free_;  // offset -> length
    // record grid (absolute indices)
    Engine::TimeGrid grid_;
    int64_t gridLoK_ = 0, gridHiK_ = -1;
    // requests
    int64_t nextId_ = 1;
    std::map<int64_t, Request> requests_;
    std::deque<int64_t> queue_;
    std::vector<int64_t> running_;
    // adaptive slice length
    double msPerObjectStep_ = 0.0;
    Stats stats_;
};

}  // namespace phop
