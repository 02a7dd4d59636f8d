// C ABI and the command-line driver of the B200 backend.
//
// The driver restates src/common/driver.cpp:57-186: the same arguments,
// validation order, error texts, exit codes and output files.
#include <cuda_runtime.h>
#include <sys/socket.h>
#include <sys/time.h>
#include <sys/un.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/parahpop.h"
#include "engine.hpp"
#include "server.hpp"

namespace fs = std::filesystem;
using phop::Value;

namespace phop {
void nrlDensityBatch(int device, int64_t n, const double* inputs, int lanes, double* outRho);  // nrl_diag.cu
}

static int g_logLevel = 1;
static thread_local std::string g_createError;

struct phop_context {
    std::unique_ptr<phop::Engine> engine;
    Value config;
    double duration = 0.0, step = 0.0;
    int64_t maxSteps = 0;
    phop::RunOptions opt;
    phop::RunStats stats;
    std::string error;
};

namespace {

// Resolve only the configuration fields documented as paths (driver.cpp:41-55).
void resolvePaths(Value& v, const fs::path& base, const std::string& key = "") {
    const bool pathField = key == "file" || key == "spaceWeatherFile" || key == "eopFile" || key == "constants"
        || key == "ephemeris" || key == "orientations";
    if (v.isString() && pathField) {
        fs::path p(v.asString());
        if (p.is_relative()) p = base / p;
        p = fs::absolute(p).lexically_normal();
        if (!fs::is_regular_file(p)) throw std::runtime_error("Required data file not found: " + p.string());
        v = Value::string(p.string());
    } else if (v.isObject()) {
        for (auto& kv : v.members()) resolvePaths(kv.second, base, kv.first);
    } else if (v.isArray()) {
        for (auto& item : v.items()) resolvePaths(item, base, key);
    }
}

void checkKeys(const Value& v, std::initializer_list<const char*> allowed, const char* context) {
    if (!v.isObject()) throw std::runtime_error(std::string(context) + " must be an object.");
    for (const auto& kv : v.members()) {
        bool found = false;
        for (const char* k : allowed) found |= kv.first == k;
        if (!found) throw std::runtime_error(std::string("Unsupported ") + context + " option: " + kv.first);
    }
}

// JSON objects written the way the reference's JSON library writes them:
// keys in sorted order.
Value sortedCopy(const Value& v) {
    if (v.isObject()) {
        Value out = Value::object();
        std::vector<std::pair<std::string, Value>> m(v.members());
        std::sort(m.begin(), m.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (auto& kv : m) out.set(kv.first, sortedCopy(kv.second));
        return out;
    }
    if (v.isArray()) {
        Value out = Value::array();
        for (auto& x : v.items()) out.push(sortedCopy(x));
        return out;
    }
    return v;
}

struct LoadedConfig {
    Value config;
    double duration = 0, step = 0;
    int64_t maxSteps = 0;
    int threads = 1;
};

// PARAHPOP_B200_SPLIT / PARAHPOP_B200_LANES: precision and lane count of the
// command-line driver's propagation
struct DriverOverrides {
    int split = -1;  // -1: library default
    int lanes = 0;   // 0: autotuned
};

DriverOverrides driverOverridesFromEnv() {
    DriverOverrides ov;
    if (const char* s = std::getenv("PARAHPOP_B200_SPLIT")) ov.split = std::atoi(s) != 0 ? 1 : 0;
    if (const char* s = std::getenv("PARAHPOP_B200_LANES")) ov.lanes = std::atoi(s);
    return ov;
}

using EngineSource = std::function<phop::Engine&(const LoadedConfig&)>;

LoadedConfig readConfig(const fs::path& configPath, const char* backend) {
    LoadedConfig lc;
    Value config = phop::parseJson(phop::readTextFile(configPath.string()));
    checkKeys(config, {"run", "execution", "model"}, "configuration");
    checkKeys(config.at("run"), {"duration_seconds"}, "run");
    checkKeys(config.at("execution"), {"maxThreads", "integration"}, "execution");
    checkKeys(config.at("execution").at("integration"), {"initialStepSize", "maxNumSteps"}, "integration");
    const int64_t maxSteps = config.at("execution").at("integration").at("maxNumSteps").asInt();
    const int64_t threads = config.at("execution").find("maxThreads") ? config.at("execution").at("maxThreads").asInt() : 1;
    if (maxSteps <= 0 || threads <= 0) throw std::runtime_error("maxNumSteps and maxThreads must be positive integers.");
    const double duration = config.at("run").at("duration_seconds").asDouble();
    config.erase("run");
    if (!(duration > 0) || !std::isfinite(duration)) throw std::runtime_error("duration_seconds must be finite and positive.");
    config.find("execution")->set("on", Value::string(backend));
    const double step = config.at("execution").at("integration").at("initialStepSize").asDouble();
    if (!(step > 0) || !std::isfinite(step)) throw std::runtime_error("initialStepSize must be finite and positive.");
    resolvePaths(config, configPath.parent_path());
    lc.config = config;
    lc.duration = duration;
    lc.step = step;
    lc.maxSteps = maxSteps;
    lc.threads = (int)threads;
    return lc;
}

}  // namespace

extern "C" {

void paraHPOP_setLogLevel(int level) { g_logLevel = level; }

int phop_create(const char* configPath, int device, phop_context** out) {
    try {
        if (!configPath || !out) throw std::runtime_error("phop_create: null argument");
        *out = nullptr;
        const fs::path cp = fs::absolute(configPath);
        LoadedConfig lc = readConfig(cp, "device");
        int count = 0;
        const cudaError_t st = cudaGetDeviceCount(&count);
        if (st != cudaSuccess || count == 0)
            throw std::runtime_error(std::string("No usable CUDA device: ") + cudaGetErrorString(st));
        phop::HostEnvironment env;
        phop::loadEnvironment(lc.config.at("model"), env);
        auto ctx = std::make_unique<phop_context>();
        ctx->engine = std::make_unique<phop::Engine>(env, device);
        ctx->config = lc.config;
        ctx->duration = lc.duration;
        ctx->step = lc.step;
        ctx->maxSteps = lc.maxSteps;
        *out = ctx.release();
        return 0;
    } catch (const std::exception& e) {
        g_createError = e.what();
        return 1;
    }
}

int phop_load_environment(const char* configPath, uint64_t* digest, double* loadMs) {
    try {
        if (!configPath) throw std::runtime_error("phop_load_environment: null argument");
        const auto t0 = std::chrono::steady_clock::now();
        LoadedConfig lc = readConfig(fs::absolute(configPath), "device");
        phop::HostEnvironment env;
        phop::loadEnvironment(lc.config.at("model"), env);
        const auto t1 = std::chrono::steady_clock::now();
        if (digest) *digest = phop::environmentDigest(env);
        if (loadMs) *loadMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
        return 0;
    } catch (const std::exception& e) {
        g_createError = e.what();
        return 1;
    }
}

void phop_destroy(phop_context* ctx) { delete ctx; }

const char* phop_last_error(const phop_context* ctx) { return ctx ? ctx->error.c_str() : g_createError.c_str(); }

int phop_run_parameters(const phop_context* ctx, double* duration, double* step, int64_t* maxSteps) {
    if (!ctx) return 1;
    if (duration) *duration = ctx->duration;
    if (step) *step = ctx->step;
    if (maxSteps) *maxSteps = ctx->maxSteps;
    return 0;
}

int phop_set_option(phop_context* ctx, const char* key, double value) {
    if (!ctx || !key) return 1;
    const std::string k(key);
    if (k == "lanes") {
        const int L = (int)value;
        if (L != 0 && L != 1 && L != 2 && L != 4 && L != 8 && L != 16) {
            ctx->error = "lanes must be 0, 1, 2, 4, 8 or 16";
            return 1;
        }
        ctx->opt.lanes = L;
    } else if (k == "split") {
        ctx->opt.split = value != 0.0;
    } else if (k == "threads") {
        const int t = (int)value;
        if (t < 32 || t > 512 || t % 32) {
            ctx->error = "threads must be a multiple of 32 in [32, 512]";
            return 1;
        }
        ctx->opt.threads = t;
    } else if (k == "ctas_per_sm") {
        ctx->opt.ctasPerSm = (int)value;
    } else if (k == "ordered") {
        ctx->opt.ordered = value != 0.0;
    } else if (k == "graph") {
        ctx->opt.graph = value != 0.0;
    } else if (k == "mixed_order") {
        const int m = (int)value;
        if (m < 0 || m > 2) {
            ctx->error = "mixed_order must be 0, 1 or 2";
            return 1;
        }
        ctx->opt.mixedOrder = m;
    } else if (k == "tile_smem") {
        ctx->opt.tileSmem = value == 0.0 ? 0 : -1;
    } else if (k == "split_floor_km") {
        if (!(value >= 0.0) || !std::isfinite(value)) {
            ctx->error = "split_floor_km must be finite and non-negative";
            return 1;
        }
        ctx->opt.splitFloorKm = value;
    } else if (k == "pair_sh") {
        if (value != -1.0 && value != 0.0 && value != 1.0) {
            ctx->error = "pair_sh must be -1 (autotuned), 0 or 1";
            return 1;
        }
        ctx->opt.pairSh = (int)value;
    } else if (k == "deep_registers") {
        if (value != -1.0 && value != 0.0 && value != 1.0) {
            ctx->error = "deep_registers must be -1 (autotuned), 0 or 1";
            return 1;
        }
        ctx->opt.deepRegs = (int)value;
    } else if (k == "tile_wait_test") {
        ctx->opt.tileWaitTest = value != 0.0 ? 1 : 0;
    } else if (k == "split_fp64_degree") {
        const int d = (int)value;
        if ((double)d != value || d < phop::kLowDeg || d > phop::kLowMax) {
            ctx->error = "split_fp64_degree must be an integer in [" + std::to_string(phop::kLowDeg) + ", "
                         + std::to_string(phop::kLowMax) + "]";
            return 1;
        }
        ctx->opt.splitFp64Degree = d;
    } else {
        ctx->error = "Unknown option: " + k;
        return 1;
    }
    return 0;
}

}  // extern "C"

namespace {

// Target arrays in the reference's target schema, checked as the driver
// checks them (driver.cpp:97-129).
phop::TargetSet makeTargets(const phop_context* ctx, int64_t n, const double* epoch, const double* states,
                            const double* mass, const double* dragArea, const double* srpArea, const double* cd,
                            const double* cr, const double* duration, const double* step) {
    if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
    if (!epoch || !states || !mass || !dragArea || !srpArea || !cd || !cr)
        throw std::runtime_error("target arrays must not be null");
    phop::TargetSet t;
    t.ids.resize(n);
    t.epoch.assign(epoch, epoch + n);
    t.state.assign(states, states + 6 * n);
    t.mass.assign(mass, mass + n);
    t.dragArea.assign(dragArea, dragArea + n);
    t.srpArea.assign(srpArea, srpArea + n);
    t.cd.assign(cd, cd + n);
    t.cr.assign(cr, cr + n);
    t.duration = duration ? std::vector<double>(duration, duration + n) : std::vector<double>(n, ctx->duration);
    t.step = step ? std::vector<double>(step, step + n) : std::vector<double>(n, ctx->step);
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 6; ++k)
            if (!std::isfinite(t.state[6 * i + k])) throw std::runtime_error("State contains a nonfinite value.");
        if (!std::isfinite(t.epoch[i]) || !std::isfinite(t.mass[i]) || !std::isfinite(t.dragArea[i])
            || !std::isfinite(t.srpArea[i]) || !std::isfinite(t.cd[i]) || !std::isfinite(t.cr[i])
            || t.mass[i] <= 0 || t.dragArea[i] <= 0 || t.srpArea[i] < 0 || t.cd[i] < 0 || t.cr[i] < 0)
            throw std::runtime_error("Invalid target epoch or physical parameter.");
        if (!(t.duration[i] > 0) || !std::isfinite(t.duration[i]))
            throw std::runtime_error("duration_seconds must be finite and positive.");
        if (!(t.step[i] > 0) || !std::isfinite(t.step[i]))
            throw std::runtime_error("initialStepSize must be finite and positive.");
    }
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        lo = std::min(lo, t.epoch[i]);
        hi = std::max(hi, t.epoch[i] + t.duration[i] / 86400.0);
    }
    ctx->engine->assertCoverage(lo, hi);
    return t;
}

}  // namespace

extern "C" {

int phop_propagate(phop_context* ctx, int64_t n, const double* epoch, const double* states, const double* mass,
                   const double* dragArea, const double* srpArea, const double* cd, const double* cr,
                   const double* duration, const double* step, double* outEpoch, double* outStates) {
    if (!ctx) return 1;
    try {
        const phop::TargetSet t = makeTargets(ctx, n, epoch, states, mass, dragArea, srpArea, cd, cr, duration, step);
        std::vector<double> oe, os;
        ctx->stats = phop::RunStats{};
        ctx->engine->propagate(t, ctx->maxSteps, ctx->opt, oe, os, &ctx->stats);
        std::copy(oe.begin(), oe.end(), outEpoch);
        std::copy(os.begin(), os.end(), outStates);
        return 0;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return 1;
    }
}

int phop_propagate_device(phop_context* ctx, int64_t n, double* dState, double epoch, const double* mass,
                          const double* dragArea, const double* srpArea, const double* cd, const double* cr,
                          double duration, double step, double* outEpoch) {
    if (!ctx) return 1;
    try {
        if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
        std::vector<double> bc(n), ams(n), ep(n, epoch);
        for (int64_t i = 0; i < n; ++i) {
            if (!(mass[i] > 0) || !(dragArea[i] > 0) || srpArea[i] < 0 || cd[i] < 0 || cr[i] < 0)
                throw std::runtime_error("Invalid target epoch or physical parameter.");
            const double area = dragArea[i] * 1e-6;
            const double crf = cr[i] * srpArea[i] / dragArea[i];
            ams[i] = crf * area / mass[i];
            bc[i] = cd[i] * area / mass[i];
        }
        ctx->engine->assertCoverage(epoch, epoch + duration / 86400.0);
        std::vector<double> oe;
        ctx->stats = phop::RunStats{};
        ctx->engine->propagateResident(n, dState, ep.data(), bc.data(), ams.data(), duration, step, ctx->maxSteps,
                                       ctx->opt, oe, &ctx->stats);
        if (outEpoch) *outEpoch = oe.empty() ? 0.0 : oe[0];
        return 0;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return 1;
    }
}

int phop_object_times(const phop_context* ctx, int64_t n, const double* epoch, const double* duration,
                      const double* step, double* outTime) {
    if (!ctx) return 1;
    phop_context* c = const_cast<phop_context*>(ctx);
    try {
        if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
        if (!epoch || !duration || !step || !outTime) throw std::runtime_error("phop_object_times: null argument");
        double lo = epoch[0], hi = epoch[0];
        for (int64_t i = 0; i < n; ++i) {
            if (!(duration[i] > 0) || !std::isfinite(duration[i]))
                throw std::runtime_error("duration_seconds must be finite and positive.");
            if (!(step[i] > 0) || !std::isfinite(step[i]))
                throw std::runtime_error("initialStepSize must be finite and positive.");
            // FixedStep.h:7-28 per object: ET epochs, first step, step count
            const double cur = std::fma(epoch[i], 86400.0, -43200.0);
            const double end = std::fma(epoch[i] + duration[i] / 86400.0, 86400.0, -43200.0);
            const double span = end - cur;
            if (!(span > 0) || !std::isfinite(span))
                throw std::runtime_error("Duration/step cannot be represented by the integration time/index types.");
            if (std::ceil(span / step[i]) > (double)c->maxSteps)
                throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
            outTime[i] = cur;
            outTime[n + i] = end;
            outTime[2 * n + i] = std::min(step[i], span);
            outTime[3 * n + i] = step[i];
            lo = std::min(lo, epoch[i]);
            hi = std::max(hi, epoch[i] + duration[i] / 86400.0);
        }
        c->engine->assertCoverage(lo, hi);
        return 0;
    } catch (const std::exception& e) {
        c->error = e.what();
        return 1;
    }
}

int phop_propagate_device_objects(phop_context* ctx, int64_t n, double* dState, double* dTime, const double* dBc,
                                  const double* dAms, int64_t maxSteps, int64_t* outUnfinished) {
    if (!ctx) return 1;
    try {
        if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
        if (!dState || !dTime || !dBc || !dAms) throw std::runtime_error("device arrays must not be null");
        ctx->stats = phop::RunStats{};
        const int64_t left = ctx->engine->advanceObjects(n, dState, dTime, dBc, dAms, maxSteps, ctx->opt, &ctx->stats);
        if (outUnfinished) *outUnfinished = left;
        return 0;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return 1;
    }
}

int phop_propagate_trajectory(phop_context* ctx, int64_t n, double epoch, const double* states, const double* mass,
                              const double* dragArea, const double* srpArea, const double* cd, const double* cr,
                              double duration, double step, int64_t every, int64_t maxRecords, double* outEpochs,
                              double* outStates, int64_t* outRecords) {
    if (!ctx) return 1;
    double* dState = nullptr;
    double* dTraj = nullptr;
    try {
        if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
        if (!states || !outEpochs || !outStates || !outRecords) throw std::runtime_error("null array argument");
        if (!(duration > 0) || !(step > 0) || !std::isfinite(duration) || !std::isfinite(step))
            throw std::runtime_error("Duration and step must be finite and positive.");
        if (every <= 0 || every > std::numeric_limits<int>::max()) throw std::runtime_error("every must be positive.");
        const int64_t steps = (int64_t)std::ceil(duration / step);
        if (steps > ctx->maxSteps) throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
        const int64_t records = steps / every;
        if (records > maxRecords) throw std::runtime_error("max_records is smaller than the trajectory's record count");
        std::vector<double> bc(n), ams(n), ep(n, epoch), soa((size_t)6 * n);
        for (int64_t i = 0; i < n; ++i) {
            if (!(mass[i] > 0) || !(dragArea[i] > 0) || srpArea[i] < 0 || cd[i] < 0 || cr[i] < 0)
                throw std::runtime_error("Invalid target epoch or physical parameter.");
            const double area = dragArea[i] * 1e-6;
            const double crf = cr[i] * srpArea[i] / dragArea[i];
            ams[i] = crf * area / mass[i];
            bc[i] = cd[i] * area / mass[i];
            for (int d = 0; d < 6; ++d) {
                if (!std::isfinite(states[6 * i + d])) throw std::runtime_error("Non-finite target state.");
                soa[(size_t)d * n + i] = states[6 * i + d];
            }
        }
        ctx->engine->assertCoverage(epoch, epoch + duration / 86400.0);
        cudaSetDevice(ctx->engine->device());
        if (cudaMalloc(&dState, soa.size() * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&dTraj, (size_t)std::max<int64_t>(records, 1) * 6 * n * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("device allocation failed for the trajectory");
        if (cudaMemcpy(dState, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("copy to the device failed");
        phop::RunOptions opt = ctx->opt;
        opt.dTraj = dTraj;
        opt.trajEvery = (int)every;
        opt.trajRecords = (int)records;
        std::vector<double> oe;
        ctx->stats = phop::RunStats{};
        ctx->engine->propagateResident(n, dState, ep.data(), bc.data(), ams.data(), duration, step, ctx->maxSteps, opt,
                                       oe, &ctx->stats);
        std::vector<double> rec((size_t)records * 6 * n);
        if (records > 0 &&
            cudaMemcpy(rec.data(), dTraj, rec.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("copy from the device failed");
        for (int64_t r = 0; r < records; ++r) {
            // record r after step (r + 1) every: t0 + k step, or the end for a
            // shortened final step
            outEpochs[r] = epoch + std::min((double)((r + 1) * every) * step, duration) / 86400.0;
            for (int64_t i = 0; i < n; ++i)
                for (int d = 0; d < 6; ++d)
                    outStates[((size_t)r * n + i) * 6 + d] = rec[((size_t)r * 6 + d) * n + i];
        }
        *outRecords = records;
        cudaFree(dState);
        cudaFree(dTraj);
        return 0;
    } catch (const std::exception& e) {
        if (dState) cudaFree(dState);
        if (dTraj) cudaFree(dTraj);
        ctx->error = e.what();
        return 1;
    }
}

int phop_propagate_device_noalloc(phop_context* ctx, int64_t n, double* dState, const double* dBc,
                                  const double* dAms, double epoch, double duration, double step, double* outEpoch) {
    if (!ctx) return 1;
    try {
        if (n <= 0) throw std::runtime_error("targets must be a nonempty array.");
        if (!dState || !dBc || !dAms) throw std::runtime_error("device arrays must not be null");
        if (!(duration > 0) || !std::isfinite(duration)) throw std::runtime_error("duration_seconds must be finite and positive.");
        if (!(step > 0) || !std::isfinite(step)) throw std::runtime_error("initialStepSize must be finite and positive.");
        ctx->engine->assertCoverage(epoch, epoch + duration / 86400.0);
        ctx->engine->propagateNoAlloc(n, dState, dBc, dAms, epoch, duration, step, ctx->maxSteps, ctx->opt, outEpoch);
        return 0;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return 1;
    }
}

// ---- serving loop ----------------------------------------------------------------------------------
}  // extern "C"

struct phop_server {
    phop_context* ctx = nullptr;
    std::unique_ptr<phop::Server> server;
    std::string error;
};

extern "C" {

int phop_server_create(phop_context* ctx, int64_t capacity, double sliceMs, phop_server** out) {
    if (!ctx || !out) return 1;
    try {
        *out = nullptr;
        auto s = std::make_unique<phop_server>();
        s->ctx = ctx;
        s->server = std::make_unique<phop::Server>(*ctx->engine, ctx->opt, capacity, sliceMs, ctx->maxSteps);
        *out = s.release();
        return 0;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return 1;
    }
}

void phop_server_destroy(phop_server* s) { delete s; }

const char* phop_server_last_error(const phop_server* s) { return s ? s->error.c_str() : ""; }

int phop_server_submit(phop_server* s, int64_t n, const double* epoch, const double* states, const double* mass,
                       const double* dragArea, const double* srpArea, const double* cd, const double* cr,
                       const double* duration, const double* step, int64_t* requestId) {
    if (!s) return 1;
    try {
        const phop::TargetSet t = makeTargets(s->ctx, n, epoch, states, mass, dragArea, srpArea, cd, cr, duration, step);
        const int64_t id = s->server->submit(t);
        if (requestId) *requestId = id;
        return 0;
    } catch (const std::exception& e) {
        s->error = e.what();
        return 1;
    }
}

int phop_server_step(phop_server* s, int64_t* finished) {
    if (!s) return 1;
    try {
        const int f = s->server->step();
        if (finished) *finished = f;
        return 0;
    } catch (const std::exception& e) {
        s->error = e.what();
        return 1;
    }
}

int phop_server_status(const phop_server* s, int64_t requestId, int* state) {
    if (!s || !state) return 1;
    try {
        *state = (int)s->server->status(requestId);
        return 0;
    } catch (const std::exception& e) {
        const_cast<phop_server*>(s)->error = e.what();
        return 1;
    }
}

int phop_server_take(phop_server* s, int64_t requestId, double* outEpoch, double* outStates, double* latencyMs,
                     double* queueMs) {
    if (!s) return 1;
    try {
        s->server->take(requestId, outEpoch, outStates, latencyMs, queueMs);
        return 0;
    } catch (const std::exception& e) {
        s->error = e.what();
        return 1;
    }
}

int phop_server_get_stats(const phop_server* s, phop_server_stats* out) {
    if (!s || !out) return 1;
    const phop::Server::Stats st = s->server->stats();
    out->queued = st.queued;
    out->running = st.running;
    out->done = st.done;
    out->failed = st.failed;
    out->active_objects = st.activeObjects;
    out->launches = st.launches;
    out->rounds = st.rounds;
    out->object_steps = st.objectSteps;
    out->busy_ms = st.busyMs;
    out->lanes = st.lanes;
    return 0;
}

int phop_last_stats(const phop_context* ctx, phop_stats* out) {
    if (!ctx || !out) return 1;
    out->kernel_ms = ctx->stats.kernelMs;
    out->records_ms = ctx->stats.recordsMs;
    out->tune_ms = ctx->stats.tuneMs;
    out->total_ms = ctx->stats.totalMs;
    out->object_steps = ctx->stats.objectSteps;
    out->launches = ctx->stats.launches;
    out->lanes = ctx->stats.lanes;
    out->ctas = ctx->stats.ctas;
    out->threads = ctx->stats.threads;
    out->split = ctx->stats.split;
    out->shared_grid = ctx->stats.sharedGrid;
    out->tile_in_smem = ctx->stats.tileInSmem;
    out->tile_fallbacks = ctx->stats.tileFallbacks;
    out->pair_sh = ctx->stats.pairSh ? 1 : 0;
    out->deep_registers = ctx->stats.deepRegs ? 1 : 0;
    out->registers = ctx->stats.registers;
    return 0;
}

}  // extern "C"

namespace {

// The driver proper, writing to `out` / `err`; `engineFor` supplies the
// device-resident environment of the loaded configuration (a fresh load for
// the in-process command line, a kept one for the resident server).
int runDriver(const std::vector<std::string>& args, const char* backend, std::ostream& out, std::ostream& err,
              const DriverOverrides& ov, const EngineSource& engineFor) {
    try {
        const int argc = (int)args.size();
        if (argc == 2 && args[1] == "--help") {
            out << "Usage: " << args[0] << " CONFIG.json TARGETS.json OUTPUT_DIRECTORY\n"
                << "Backend: " << backend << "; integrator: RKF78 fixed step\n";
            return 0;
        }
        if (argc != 4) throw std::runtime_error("Expected CONFIG.json TARGETS.json OUTPUT_DIRECTORY (or --help).");
        const fs::path configPath = fs::absolute(args[1]);
        const fs::path inputPath = fs::absolute(args[2]);
        const fs::path outputPath = fs::absolute(args[3]);
        for (const char* f : {"final_states.csv", "summary.json", "configuration_resolved.json"})
            if (fs::exists(outputPath / f))
                throw std::runtime_error("Output exists; use a new directory: " + outputPath.string());
        LoadedConfig lc = readConfig(configPath, backend);
        const Value input = phop::parseJson(phop::readTextFile(inputPath.string()));
        const Value& targets = input.at("targets");
        if (!targets.isArray() || targets.size() == 0) throw std::runtime_error("targets must be a nonempty array.");
        if (targets.size() > (size_t)std::numeric_limits<int32_t>::max())
            throw std::runtime_error("Too many targets for the engine index type.");
        const int64_t n = (int64_t)targets.size();
        phop::TargetSet t;
        std::set<int64_t> ids;
        double earliest = INFINITY, latest = -INFINITY;
        for (int64_t i = 0; i < n; ++i) {
            const Value& tg = targets[i];
            const int64_t id = tg.at("id").asInt();
            if (!ids.insert(id).second) throw std::runtime_error("Target IDs must be unique.");
            const Value& st = tg.at("state_km_km_s");
            if (!st.isArray() || st.size() != 6) throw std::runtime_error("state_km_km_s must hold six numbers.");
            for (int k = 0; k < 6; ++k) {
                const double x = st[k].asDouble();
                if (!std::isfinite(x)) throw std::runtime_error("State contains a nonfinite value.");
                t.state.push_back(x);
            }
            const double epoch = tg.at("epoch_mjd2000_tdb").asDouble();
            const double mass = tg.at("mass_kg").asDouble();
            const double area = tg.at("drag_area_m2").asDouble();
            const double srp = tg.at("srp_area_m2").asDouble();
            const double cd = tg.at("cd").asDouble();
            const double cr = tg.at("cr").asDouble();
            if (!std::isfinite(epoch) || !std::isfinite(mass) || !std::isfinite(area) || !std::isfinite(srp)
                || !std::isfinite(cd) || !std::isfinite(cr) || mass <= 0 || area <= 0 || srp < 0 || cd < 0 || cr < 0)
                throw std::runtime_error("Invalid target epoch or physical parameter.");
            // per-target duration / step: extension for mixed populations
            const double dur = tg.numberOr("duration_seconds", lc.duration);
            const double stp = tg.numberOr("step_seconds", lc.step);
            if (!(dur > 0) || !std::isfinite(dur)) throw std::runtime_error("duration_seconds must be finite and positive.");
            if (!(stp > 0) || !std::isfinite(stp)) throw std::runtime_error("initialStepSize must be finite and positive.");
            t.ids.push_back(id);
            t.epoch.push_back(epoch);
            t.mass.push_back(mass);
            t.dragArea.push_back(area);
            t.srpArea.push_back(srp);
            t.cd.push_back(cd);
            t.cr.push_back(cr);
            t.duration.push_back(dur);
            t.step.push_back(stp);
            earliest = std::min(earliest, epoch);
            latest = std::max(latest, epoch + dur / 86400.0);
        }
        if (std::string(backend) == "device") {
            int count = 0;
            const cudaError_t status = cudaGetDeviceCount(&count);
            if (status != cudaSuccess || count == 0)
                throw std::runtime_error(std::string("No usable CUDA device: ") + cudaGetErrorString(status));
        }
        const auto environmentStart = std::chrono::steady_clock::now();
        phop::Engine& engine = engineFor(lc);
        engine.assertCoverage(earliest, latest);
        const auto integrationStart = std::chrono::steady_clock::now();
        std::vector<double> finalEpoch, finalState;
        phop::RunOptions opt;
        if (ov.split >= 0) opt.split = ov.split != 0;
        opt.lanes = ov.lanes;
        engine.propagate(t, lc.maxSteps, opt, finalEpoch, finalState, nullptr);
        {
            const cudaError_t status = cudaDeviceSynchronize();
            if (status != cudaSuccess) throw std::runtime_error(cudaGetErrorString(status));
        }
        const auto integrationEnd = std::chrono::steady_clock::now();
        double maxEpochError = 0;
        for (int64_t i = 0; i < n; ++i) {
            const double expected = t.epoch[i] + t.duration[i] / 86400.0;
            const double err = std::abs(finalEpoch[i] - expected) * 86400.0;
            if (!std::isfinite(err) || err > 1e-4) throw std::runtime_error("A target did not reach its requested end epoch.");
            maxEpochError = std::max(maxEpochError, err);
            for (int k = 0; k < 6; ++k)
                if (!std::isfinite(finalState[6 * i + k])) throw std::runtime_error("Nonfinite final state.");
        }
        fs::create_directories(outputPath);
        std::ofstream csv(outputPath / "final_states.csv");
        csv << "id,epoch_mjd2000_tdb,x_km,y_km,z_km,vx_km_s,vy_km_s,vz_km_s\n" << std::setprecision(17);
        for (int64_t i = 0; i < n; ++i) {
            csv << t.ids[i] << ',' << finalEpoch[i];
            for (int k = 0; k < 6; ++k) csv << ',' << finalState[6 * i + k];
            csv << '\n';
        }
        csv.close();
        if (!csv) throw std::runtime_error("Failed to write final_states.csv.");
        Value summary = Value::object();
        summary.set("backend", Value::string(backend));
        summary.set("targets", Value::integer(n));
        summary.set("integrator", Value::string("RKF78 fixed step"));
        summary.set("initial_step_seconds", Value::real(lc.step));
        summary.set("duration_seconds", Value::real(lc.duration));
        summary.set("environment_seconds",
                    Value::real(std::chrono::duration<double>(integrationStart - environmentStart).count()));
        summary.set("propagation_seconds",
                    Value::real(std::chrono::duration<double>(integrationEnd - integrationStart).count()));
        summary.set("max_end_epoch_error_seconds", Value::real(maxEpochError));
        summary.set("validation_passed", Value::boolean(true));
        std::ofstream resolved(outputPath / "configuration_resolved.json");
        resolved << sortedCopy(lc.config).dump(2) << '\n';
        resolved.close();
        if (!resolved) throw std::runtime_error("Failed to write resolved configuration.");
        const std::string sj = sortedCopy(summary).dump(2);
        std::ofstream ss(outputPath / "summary.json");
        ss << sj << '\n';
        ss.close();
        if (!ss) throw std::runtime_error("Failed to write summary.");
        out << sj << '\n';
        return 0;
    } catch (const std::exception& e) {
        err << "ParaHPOP: " << e.what() << '\n';
        return 1;
    }
}


// ---- resident environment server -------------------------------------------
// `parahpop_gpu --serve SOCKET` keeps environments resident on the device
// between command-line runs: a client run (PARAHPOP_B200_SERVER=SOCKET
// parahpop_gpu CONFIG TARGETS OUTPUT) sends its three absolute paths over a
// Unix-domain socket, the server runs the driver with a kept environment
// when the configuration's model section and the size and modification time
// of every file it names are unchanged (a fresh load otherwise), writes the
// output files itself and returns the exit status and the text of standard
// output and error, which the client prints.  Requests are served one at a
// time.  Messages: a 4-byte little-endian length, then JSON.

constexpr size_t kResidentMaxMessage = size_t(64) << 20;
constexpr size_t kResidentKeep = 4;  // environments kept (least recently used evicted)

bool ioAll(int fd, void* buf, size_t n, bool writing) {
    char* p = (char*)buf;
    while (n > 0) {
        const ssize_t k = writing ? ::send(fd, p, n, MSG_NOSIGNAL) : ::recv(fd, p, n, 0);
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0) return false;
        p += k;
        n -= (size_t)k;
    }
    return true;
}

bool sendMessage(int fd, const std::string& text) {
    if (text.size() > kResidentMaxMessage) return false;
    unsigned char len[4];
    for (int i = 0; i < 4; ++i) len[i] = (unsigned char)((text.size() >> (8 * i)) & 0xff);
    return ioAll(fd, len, 4, true) && ioAll(fd, (void*)text.data(), text.size(), true);
}

bool receiveMessage(int fd, std::string& text) {
    unsigned char len[4];
    if (!ioAll(fd, len, 4, false)) return false;
    size_t n = 0;
    for (int i = 0; i < 4; ++i) n |= (size_t)len[i] << (8 * i);
    if (n > kResidentMaxMessage) return false;
    text.assign(n, '\0');
    return n == 0 || ioAll(fd, &text[0], n, false);
}

// socket address of `path`; false when the path does not fit
bool socketAddress(const std::string& path, sockaddr_un& addr) {
    std::memset(&addr, 0, sizeof(addr));
    addr.sun_family = AF_UNIX;
    if (path.empty() || path.size() >= sizeof(addr.sun_path)) return false;
    std::memcpy(addr.sun_path, path.c_str(), path.size());
    return true;
}

int connectTo(const std::string& path, std::string& why) {
    sockaddr_un addr;
    if (!socketAddress(path, addr)) {
        why = "socket path is empty or too long";
        return -1;
    }
    const int fd = ::socket(AF_UNIX, SOCK_STREAM, 0);
    if (fd < 0) {
        why = std::strerror(errno);
        return -1;
    }
    if (::connect(fd, (const sockaddr*)&addr, sizeof(addr)) != 0) {
        why = std::strerror(errno);
        ::close(fd);
        return -1;
    }
    return fd;
}

// The data files a resolved model section names, with size and modification
// time: part of the key under which the server keeps its environment.
void fileStamps(const Value& v, std::string& key) {
    if (v.isString()) {
        std::error_code ec;
        const fs::path p(v.asString());
        if (p.is_absolute() && fs::is_regular_file(p, ec)) {
            const auto size = fs::file_size(p, ec);
            const auto mtime = fs::last_write_time(p, ec).time_since_epoch().count();
            key += "\n" + p.string() + "|" + std::to_string(size) + "|" + std::to_string((long long)mtime);
        }
    } else if (v.isObject()) {
        for (const auto& kv : v.members()) fileStamps(kv.second, key);
    } else if (v.isArray()) {
        for (const auto& item : v.items()) fileStamps(item, key);
    }
}

struct KeptEnvironment {
    std::string key;
    std::unique_ptr<phop::Engine> engine;
    uint64_t lastUse = 0;
};

int residentServe(const std::string& path, const char* backend) {
    sockaddr_un addr;
    if (!socketAddress(path, addr)) {
        std::cerr << "ParaHPOP: socket path is empty or too long: " << path << '\n';
        return 1;
    }
    {
        std::string why;
        const int probe = connectTo(path, why);
        if (probe >= 0) {
            ::close(probe);
            std::cerr << "ParaHPOP: a server already answers at " << path << '\n';
            return 1;
        }
    }
    std::error_code ec;
    if (fs::is_socket(path, ec)) fs::remove(path, ec);  // left behind by a server that did not stop cleanly
    const int lfd = ::socket(AF_UNIX, SOCK_STREAM, 0);
    if (lfd < 0 || ::bind(lfd, (const sockaddr*)&addr, sizeof(addr)) != 0 || ::listen(lfd, 16) != 0) {
        std::cerr << "ParaHPOP: cannot listen at " << path << ": " << std::strerror(errno) << '\n';
        if (lfd >= 0) ::close(lfd);
        return 1;
    }
    std::cout << "ParaHPOP: resident environment server listening at " << path << std::endl;
    std::vector<KeptEnvironment> kept;
    uint64_t clock = 0;
    int status = 0;
    for (bool serving = true; serving;) {
        const int fd = ::accept(lfd, nullptr, nullptr);
        if (fd < 0) {
            if (errno == EINTR) continue;
            std::cerr << "ParaHPOP: accept failed: " << std::strerror(errno) << '\n';
            status = 1;
            break;
        }
        timeval tv{30, 0};  // a client that stops talking does not hold the server
        ::setsockopt(fd, SOL_SOCKET, SO_RCVTIMEO, &tv, sizeof(tv));
        std::string request;
        Value reply = Value::object();
        try {
            if (!receiveMessage(fd, request)) throw std::runtime_error("incomplete request");
            const Value req = phop::parseJson(request);
            if (const Value* stop = req.find("stop"); stop && stop->asBool()) {
                reply.set("status", Value::integer(0));
                reply.set("stdout", Value::string(""));
                reply.set("stderr", Value::string(""));
                serving = false;
            } else {
                std::vector<std::string> args{"parahpop_gpu"};
                for (const Value& a : req.at("args").items()) args.push_back(a.asString());
                DriverOverrides ov;
                ov.split = (int)req.at("split").asInt();
                ov.lanes = (int)req.at("lanes").asInt();
                std::ostringstream out, err;
                const int rc = runDriver(args, backend, out, err, ov, [&](const LoadedConfig& lc) -> phop::Engine& {
                    const Value& model = lc.config.at("model");
                    std::string key = model.dump();
                    fileStamps(model, key);
                    for (auto& k : kept)
                        if (k.key == key) {
                            k.lastUse = ++clock;
                            return *k.engine;
                        }
                    phop::HostEnvironment env;
                    phop::loadEnvironment(model, env);
                    if (kept.size() >= kResidentKeep) {
                        auto lru = std::min_element(kept.begin(), kept.end(),
                                                    [](const auto& a, const auto& b) { return a.lastUse < b.lastUse; });
                        kept.erase(lru);
                    }
                    kept.push_back(KeptEnvironment{key, std::make_unique<phop::Engine>(env, 0), ++clock});
                    return *kept.back().engine;
                });
                reply.set("status", Value::integer(rc));
                reply.set("stdout", Value::string(out.str()));
                reply.set("stderr", Value::string(err.str()));
                // a device error leaves the context unusable: answer, then stop
                const cudaError_t dev = cudaDeviceSynchronize();
                if (dev != cudaSuccess && dev != cudaErrorNoDevice && dev != cudaErrorInsufficientDriver) {
                    std::cerr << "ParaHPOP: device error, server stops: " << cudaGetErrorString(dev) << '\n';
                    status = 1;
                    serving = false;
                }
            }
        } catch (const std::exception& e) {
            reply.set("status", Value::integer(1));
            reply.set("stdout", Value::string(""));
            reply.set("stderr", Value::string(std::string("ParaHPOP: ") + e.what() + "\n"));
        }
        sendMessage(fd, reply.dump());
        ::close(fd);
    }
    ::close(lfd);
    fs::remove(path, ec);
    kept.clear();
    return status;
}

int residentClient(const std::string& path, const std::vector<std::string>& args, const DriverOverrides& ov) {
    std::string why;
    const int fd = connectTo(path, why);
    if (fd < 0) {
        std::cerr << "ParaHPOP: no resident environment server answers at " << path << ": " << why << '\n';
        return 1;
    }
    Value req = Value::object();
    Value a = Value::array();
    for (size_t i = 1; i < args.size(); ++i) a.push(Value::string(fs::absolute(args[i]).string()));
    req.set("args", a);
    req.set("split", Value::integer(ov.split));
    req.set("lanes", Value::integer(ov.lanes));
    std::string text;
    const bool ok = sendMessage(fd, req.dump()) && receiveMessage(fd, text);
    ::close(fd);
    if (!ok) {
        std::cerr << "ParaHPOP: the resident environment server at " << path << " did not answer.\n";
        return 1;
    }
    try {
        const Value reply = phop::parseJson(text);
        std::cout << reply.at("stdout").asString();
        std::cerr << reply.at("stderr").asString();
        return (int)reply.at("status").asInt();
    } catch (const std::exception& e) {
        std::cerr << "ParaHPOP: malformed answer from the resident environment server: " << e.what() << '\n';
        return 1;
    }
}

int residentStop(const std::string& path) {
    std::string why;
    const int fd = connectTo(path, why);
    if (fd < 0) return 1;
    Value req = Value::object();
    req.set("stop", Value::boolean(true));
    std::string text;
    const bool ok = sendMessage(fd, req.dump()) && receiveMessage(fd, text);
    ::close(fd);
    return ok ? 0 : 1;
}


}  // namespace

extern "C" {

int paraHPOP_run(int argc, char** argv, const char* backend) {
    std::vector<std::string> args(argv, argv + argc);
    const DriverOverrides ov = driverOverridesFromEnv();
    const char* server = std::getenv("PARAHPOP_B200_SERVER");
    if (server && *server && argc == 4) return residentClient(server, args, ov);
    std::unique_ptr<phop::Engine> engine;
    return runDriver(args, backend, std::cout, std::cerr, ov, [&](const LoadedConfig& lc) -> phop::Engine& {
        phop::HostEnvironment env;
        phop::loadEnvironment(lc.config.at("model"), env);
        engine = std::make_unique<phop::Engine>(env, 0);
        return *engine;
    });
}

int phop_resident_serve(const char* socket_path, const char* backend) {
    return residentServe(socket_path ? socket_path : "", backend ? backend : "device");
}

int phop_resident_stop(const char* socket_path) { return residentStop(socket_path ? socket_path : ""); }

int phop_nrlmsise00_density(int device, int64_t n, const double* inputs, int lanes, double* out_rho) {
    try {
        phop::nrlDensityBatch(device, n, inputs, lanes, out_rho);
        g_createError.clear();
        return 0;
    } catch (const std::exception& e) {
        g_createError = e.what();
        return 1;
    }
}

}  // extern "C"
