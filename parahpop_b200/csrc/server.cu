// Serving loop (server.hpp): object pool, admission, slices and retirement.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include "server.hpp"

namespace phop {

#define PHOP_SCUDA(call)                                                                                   \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_)); \
    } while (0)

namespace {
// FixedStep.h:7-37 time conventions (TDB seconds past J2000 noon)
double mjdToEtS(double mjd) { return std::fma(mjd, 86400.0, -43200.0); }
double etToMjdS(double et) { return std::fma(et, 1.0 / 86400.0, 0.5); }
constexpr int64_t kGridMarginPoints = 2880;   // 24 h of 30 s records built ahead
constexpr int64_t kGridMaxPoints = int64_t(1) << 22;
constexpr int64_t kMinActive = 65536;          // objects that keep every SM busy
}  // namespace

Server::Server(Engine& engine, const RunOptions& opt, int64_t capacity, double sliceMs, int64_t maxSteps)
    : engine_(engine), opt_(opt), capacity_(capacity), sliceMs_(sliceMs), maxSteps_(maxSteps) {
    if (capacity <= 0 || capacity > (int64_t)INT32_MAX) throw std::runtime_error("server capacity must be in [1, 2^31)");
    if (!(sliceMs > 0) || !std::isfinite(sliceMs)) throw std::runtime_error("slice_ms must be finite and positive");
    // one lane split for the server's lifetime keeps every object's arithmetic
    // independent of its batch-mates
    lanes_ = opt.lanes > 0 ? opt.lanes : 2;
    PHOP_SCUDA(cudaSetDevice(engine.device()));
    PHOP_SCUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    PHOP_SCUDA(cudaEventCreate(&ev0_));
    PHOP_SCUDA(cudaEventCreate(&ev1_));
    const size_t C = (size_t)capacity;
    PHOP_SCUDA(cudaMalloc(&state_, 6 * C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&bc_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&ams_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&cur_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&end_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&dt_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&step_, C * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&unfinished_, C * sizeof(int)));
    PHOP_SCUDA(cudaMalloc(&active_, C * sizeof(int64_t)));
    PHOP_SCUDA(cudaMalloc(&ctl_, 2 * sizeof(int)));
    PHOP_SCUDA(cudaMemset(unfinished_, 0, C * sizeof(int)));
    hostUnfinished_.assign(C, 0);
    free_[0] = capacity;
    stats_.lanes = lanes_;
}

Server::~Server() {
    cudaSetDevice(engine_.device());
    if (stream_) cudaStreamSynchronize(stream_);
    for (void* p : {(void*)state_, (void*)bc_, (void*)ams_, (void*)cur_, (void*)end_, (void*)dt_, (void*)step_,
                    (void*)unfinished_, (void*)active_, (void*)ctl_, (void*)grid_.grid, (void*)grid_.gridPairs})
        if (p) cudaFree(p);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

// first fit over the free ranges
bool Server::allocate(int64_t n, int64_t& off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second >= n) {
            off = it->first;
            const int64_t rest = it->second - n;
            free_.erase(it);
            if (rest > 0) free_[off + n] = rest;
            return true;
        }
    }
    return false;
}

void Server::release(int64_t off, int64_t n) {
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
        it->second += next->second;
        free_.erase(next);
    }
    if (it != free_.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            free_.erase(it);
        }
    }
}

int64_t Server::submit(const TargetSet& t) {
    const int64_t n = (int64_t)t.size();
    if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
    if (n > capacity_) throw std::runtime_error("request of " + std::to_string(n) + " objects exceeds the server capacity of "
                                                + std::to_string(capacity_));
    Request r;
    r.id = nextId_++;
    r.t = t;
    r.lo = INFINITY;
    r.hi = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        const double a = mjdToEtS(t.epoch[i]);
        const double b = mjdToEtS(t.epoch[i] + t.duration[i] / 86400.0);
        const double span = b - a;
        if (!(span > 0) || !std::isfinite(span))
            throw std::runtime_error("Duration/step cannot be represented by the integration time/index types.");
        r.objectSteps += (int64_t)std::ceil(span / t.step[i]);
        r.lo = std::min(r.lo, a);
        r.hi = std::max(r.hi, b);
    }
    r.submitted = std::chrono::steady_clock::now();
    const int64_t id = r.id;
    requests_.emplace(id, std::move(r));
    queue_.push_back(id);
    return id;
}

void Server::admit(Request& r) {
    const int64_t n = (int64_t)r.t.size(), off = r.off, C = capacity_;
    std::vector<double> soa((size_t)6 * n), bc(n), ams(n), cur(n), end(n), dt(n), stp(n);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < 6; ++d) soa[(size_t)d * n + i] = r.t.state[(size_t)6 * i + d];
        // driver.cpp:118-120 then PrivateAccelerations.h:41-42
        const double area = r.t.dragArea[i] * 1e-6;
        const double crf = r.t.cr[i] * r.t.srpArea[i] / r.t.dragArea[i];
        ams[i] = crf * area / r.t.mass[i];
        bc[i] = r.t.cd[i] * area / r.t.mass[i];
        cur[i] = mjdToEtS(r.t.epoch[i]);
        end[i] = mjdToEtS(r.t.epoch[i] + r.t.duration[i] / 86400.0);
        dt[i] = std::min(r.t.step[i], end[i] - cur[i]);
        stp[i] = r.t.step[i];
    }
    const size_t nb = (size_t)n * sizeof(double);
    for (int d = 0; d < 6; ++d)
        PHOP_SCUDA(cudaMemcpyAsync(state_ + (size_t)d * C + off, soa.data() + (size_t)d * n, nb, cudaMemcpyHostToDevice,
                                   stream_));
    PHOP_SCUDA(cudaMemcpyAsync(bc_ + off, bc.data(), nb, cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaMemcpyAsync(ams_ + off, ams.data(), nb, cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaMemcpyAsync(cur_ + off, cur.data(), nb, cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaMemcpyAsync(end_ + off, end.data(), nb, cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaMemcpyAsync(dt_ + off, dt.data(), nb, cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaMemcpyAsync(step_ + off, stp.data(), nb, cudaMemcpyHostToDevice, stream_));
    std::vector<int> ones(n, 1);
    PHOP_SCUDA(cudaMemcpyAsync(unfinished_ + off, ones.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, stream_));
    PHOP_SCUDA(cudaStreamSynchronize(stream_));
    std::fill(hostUnfinished_.begin() + off, hostUnfinished_.begin() + off + n, 1);
    r.state = Running;
    r.admitted = std::chrono::steady_clock::now();
}

void Server::finish(Request& r) {
    const int64_t n = (int64_t)r.t.size(), off = r.off, C = capacity_;
    std::vector<double> soa((size_t)6 * n), cur(n);
    const size_t nb = (size_t)n * sizeof(double);
    for (int d = 0; d < 6; ++d)
        PHOP_SCUDA(cudaMemcpyAsync(soa.data() + (size_t)d * n, state_ + (size_t)d * C + off, nb, cudaMemcpyDeviceToHost,
                                   stream_));
    PHOP_SCUDA(cudaMemcpyAsync(cur.data(), cur_ + off, nb, cudaMemcpyDeviceToHost, stream_));
    PHOP_SCUDA(cudaStreamSynchronize(stream_));
    r.outState.assign((size_t)6 * n, 0.0);
    r.outEpoch.assign(n, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < 6; ++d) r.outState[(size_t)6 * i + d] = soa[(size_t)d * n + i];
        r.outEpoch[i] = etToMjdS(cur[i]);
    }
    release(off, n);
    r.state = Done;
    r.finished = std::chrono::steady_clock::now();
    r.t = TargetSet{};
    stats_.objectSteps += r.objectSteps;
    ++stats_.done;
}

void Server::ensureGrid(double lo, double hi) {
    const double H = kRecordGridSeconds;
    const int64_t kLo = (int64_t)std::floor(lo / H) - 1;
    const int64_t kHi = (int64_t)std::ceil(hi / H) + 2;
    if (grid_.grid && kLo >= gridLoK_ && kHi <= gridHiK_) return;
    int64_t a = kLo, b = kHi + kGridMarginPoints;
    if (grid_.grid && std::max(b, gridHiK_) - std::min(a, gridLoK_) + 1 <= kGridMaxPoints) {
        a = std::min(a, gridLoK_);
        b = std::max(b, gridHiK_);
    }
    const int64_t G = b - a + 1;
    if (G > kGridMaxPoints) throw std::runtime_error("the admitted requests span too long a time interval");
    std::vector<double> ts(G);
    for (int64_t k = 0; k < G; ++k) ts[k] = (double)(a + k) * H;
    double* dT = nullptr;
    EpochRecord* rec = nullptr;
    PHOP_SCUDA(cudaStreamSynchronize(stream_));
    if (grid_.grid) cudaFree((void*)grid_.grid);
    if (grid_.gridPairs) cudaFree((void*)grid_.gridPairs);
    grid_.grid = nullptr;
    grid_.gridPairs = nullptr;
    PHOP_SCUDA(cudaMalloc(&dT, (size_t)G * sizeof(double)));
    PHOP_SCUDA(cudaMalloc(&rec, (size_t)G * sizeof(EpochRecord)));
    PHOP_SCUDA(cudaMemcpyAsync(dT, ts.data(), (size_t)G * sizeof(double), cudaMemcpyHostToDevice, stream_));
    launchEpochRecords(engine_.denv_, dT, (int)G, rec, stream_);
    PHOP_SCUDA(cudaGetLastError());
    double2* pairs = nullptr;
    PHOP_SCUDA(cudaMalloc(&pairs, (size_t)(G - 1) * kInterpFields * sizeof(double2)));
    launchRecordPairs(rec, G, pairs, stream_);
    PHOP_SCUDA(cudaGetLastError());
    ++stats_.launches;
    PHOP_SCUDA(cudaStreamSynchronize(stream_));
    cudaFree(dT);
    ++stats_.launches;
    grid_.grid = rec;
    grid_.gridPairs = pairs;
    grid_.gridH = H;
    grid_.gridBase = a;
    grid_.gridN = (int)G;
    gridLoK_ = a;
    gridHiK_ = b;
}

int Server::step() {
    PHOP_SCUDA(cudaSetDevice(engine_.device()));
    ++stats_.rounds;
    // admission: first come first served, later requests may fill gaps the
    // head of the queue does not fit.  Two budgets: pool slots (HBM) and
    // compute - the unfinished objects of the running batch are kept to what
    // one step of the measured rate covers in a slice (at least kMinActive,
    // so the GPU stays full), which bounds how long a newly admitted request
    // shares each slice with the rest; a request above that limit is
    // admitted when nothing else runs.
    int64_t active = 0;
    for (int64_t id : running_) {
        const Request& r = requests_.at(id);
        for (int64_t i = 0; i < (int64_t)r.t.size(); ++i) active += hostUnfinished_[r.off + i];
    }
    const int64_t computeLimit =
        msPerObjectStep_ > 0 ? std::max<int64_t>(kMinActive, (int64_t)(sliceMs_ / msPerObjectStep_)) : capacity_;
    for (auto it = queue_.begin(); it != queue_.end();) {
        Request& r = requests_.at(*it);
        const int64_t n = (int64_t)r.t.size();
        int64_t off = 0;
        if ((active + n <= computeLimit || active == 0) && allocate(n, off)) {
            active += n;
            r.off = off;
            admit(r);
            running_.push_back(r.id);
            it = queue_.erase(it);
        } else {
            ++it;
        }
    }
    if (running_.empty()) return 0;
    std::vector<int64_t> act;
    double lo = INFINITY, hi = -INFINITY;
    int64_t allowance = INT64_MAX;
    for (int64_t id : running_) {
        const Request& r = requests_.at(id);
        const int64_t n = (int64_t)r.t.size();
        for (int64_t i = 0; i < n; ++i)
            if (hostUnfinished_[r.off + i]) act.push_back(r.off + i);
        lo = std::min(lo, r.lo);
        hi = std::max(hi, r.hi);
        allowance = std::min(allowance, maxSteps_ - r.steps);
    }
    const int64_t nAct = (int64_t)act.size();
    int64_t K = 0;
    if (nAct > 0) {
        // steps in this slice: the target slice length at the measured cost
        K = msPerObjectStep_ > 0 ? (int64_t)(sliceMs_ / (msPerObjectStep_ * (double)nAct)) : 8;
        K = std::max<int64_t>(1, std::min<int64_t>(K, 1 << 20));
        K = std::min(K, std::max<int64_t>(allowance, 1));
        PHOP_SCUDA(cudaMemcpyAsync(active_, act.data(), (size_t)nAct * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        int64_t launches = 0;
        const int64_t* order = opt_.ordered ? engine_.orderByRadius(nAct, state_, stream_, &launches, capacity_, active_)
                                            : active_;
        ensureGrid(lo, hi);
        StepParams p{};
        p.env = engine_.denv_;
        p.n = nAct;
        p.state = state_;
        p.bc = bc_;
        p.ams = ams_;
        p.low = engine_.dLow_;
        p.diagC = engine_.dDiag_;
        p.maxSteps = K;
        p.order = order;
        p.cur = cur_;
        p.end = end_;
        p.dt = dt_;
        p.step = step_;
        p.unfinished = unfinished_;
        p.grid = grid_.grid;
        p.gridPairs = grid_.gridPairs;
        p.gridH = grid_.gridH;
        p.gridBase = grid_.gridBase;
        p.gridN = grid_.gridN;
        p.stride = capacity_;
        p.workCounter = ctl_;
        p.errorFlag = ctl_ + 1;
        PHOP_SCUDA(cudaEventRecord(ev0_, stream_));
        engine_.launchStep(p, lanes_, opt_, false, stream_);
        PHOP_SCUDA(cudaEventRecord(ev1_, stream_));
        PHOP_SCUDA(cudaEventSynchronize(ev1_));
        launches += 1;
        stats_.launches += launches;
        int err = 0;
        PHOP_SCUDA(cudaMemcpy(&err, ctl_ + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) throw std::runtime_error("Propagation kernel reported error " + std::to_string(err) + ".");
        float ms = 0.f;
        PHOP_SCUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
        stats_.busyMs += ms;
        const double per = (double)ms / ((double)K * (double)nAct);
        msPerObjectStep_ = msPerObjectStep_ > 0 ? 0.5 * (msPerObjectStep_ + per) : per;
        const int64_t top = *std::max_element(act.begin(), act.end()) + 1;
        PHOP_SCUDA(cudaMemcpy(hostUnfinished_.data(), unfinished_, (size_t)top * sizeof(int), cudaMemcpyDeviceToHost));
    }
    int finished = 0;
    std::vector<int64_t> still;
    for (int64_t id : running_) {
        Request& r = requests_.at(id);
        r.steps += K;
        const int64_t n = (int64_t)r.t.size();
        bool all = true;
        for (int64_t i = 0; i < n && all; ++i) all = hostUnfinished_[r.off + i] == 0;
        if (all) {
            finish(r);
            ++finished;
        } else if (r.steps >= maxSteps_) {
            release(r.off, n);
            std::fill(hostUnfinished_.begin() + r.off, hostUnfinished_.begin() + r.off + n, 0);
            r.state = Failed;
            r.error = "A target stopped without reaching the requested end of simulation.";
            r.finished = std::chrono::steady_clock::now();
            r.t = TargetSet{};
            ++stats_.failed;
            ++finished;
        } else {
            still.push_back(id);
        }
    }
    running_.swap(still);
    // unfinished objects of the requests still running
    int64_t remaining = 0;
    for (int64_t id : running_) {
        const Request& r = requests_.at(id);
        for (int64_t i = 0; i < (int64_t)r.t.size(); ++i) remaining += hostUnfinished_[r.off + i];
    }
    stats_.activeObjects = remaining;
    return finished;
}

Server::State Server::status(int64_t id) const {
    auto it = requests_.find(id);
    if (it == requests_.end()) throw std::runtime_error("unknown request id " + std::to_string(id));
    return it->second.state;
}

void Server::take(int64_t id, double* outEpoch, double* outStates, double* latencyMs, double* queueMs) {
    auto it = requests_.find(id);
    if (it == requests_.end()) throw std::runtime_error("unknown request id " + std::to_string(id));
    Request& r = it->second;
    if (r.state == Queued || r.state == Running) throw std::runtime_error("request " + std::to_string(id) + " has not finished");
    const auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    if (latencyMs) *latencyMs = ms(r.submitted, r.finished);
    if (queueMs) *queueMs = r.state == Done ? ms(r.submitted, r.admitted) : 0.0;
    if (r.state == Failed) {
        const std::string e = r.error;
        requests_.erase(it);
        throw std::runtime_error(e);
    }
    if (outEpoch) std::copy(r.outEpoch.begin(), r.outEpoch.end(), outEpoch);
    if (outStates) std::copy(r.outState.begin(), r.outState.end(), outStates);
    requests_.erase(it);
}

Server::Stats Server::stats() const {
    Stats s = stats_;
    s.queued = (int64_t)queue_.size();
    s.running = (int64_t)running_.size();
    return s;
}

}  // namespace phop
