/*
 * parahpop-b200 C ABI: the drop-in boundary of the B200 propagation backend.
 *
 * Shared library: parahpop_b200/lib/libparahpop_engine.so
 * Command line:   parahpop_b200/bin/parahpop_gpu CONFIG.json TARGETS.json OUTPUT_DIRECTORY
 *
 * Conventions: plain C types only; every call returns 0 on success and 1 on
 * failure (the reference driver's exit codes); the failure text is available
 * from phop_last_error().  The library owns device memory; callers own every
 * host buffer they pass.  One context holds one loaded model configuration
 * resident on one GPU and is used by one host thread at a time.
 *
 * Units and frames are the reference's: states in km and km/s in Earth-centred
 * ICRF-aligned axes, epochs in MJD2000 TDB days, areas in m^2, masses in kg.
 */
#ifndef PARAHPOP_B200_H
#define PARAHPOP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct phop_context phop_context;

/* Replaces the reference export of the same name and signature
 * (src/common/engine/paraHPOP/util/log.cu:26-38): 0 silences informational
 * output, higher values enable it. */
void paraHPOP_setLogLevel(int level);

/* The reference command-line driver, in process: argument and JSON checks,
 * environment load, propagation, final_states.csv / summary.json /
 * configuration_resolved.json outputs, "ParaHPOP: <message>" on stderr and
 * exit status 0/1.  Replaces int paraHPOP::run(int, char**, const char*)
 * (include/paraHPOP/driver.h:3, src/common/driver.cpp:57-186); `backend` is
 * reported in summary.json ("device" for parahpop_gpu). */
int paraHPOP_run(int argc, char** argv, const char* backend);

/* ---- resident environment across command-line runs (no counterpart in the
 * reference, whose driver loads and uploads the environment in every run,
 * src/common/driver.cpp:132-135) ------------------------------------------
 * phop_resident_serve listens on the Unix-domain socket `socket_path` and
 * serves command-line runs one at a time until phop_resident_stop: a run of
 * paraHPOP_run with PARAHPOP_B200_SERVER=<socket_path> in its environment
 * (CONFIG TARGETS OUTPUT form) sends its absolute paths and the
 * PARAHPOP_B200_SPLIT / PARAHPOP_B200_LANES settings to the server, which
 * runs the driver there -- same checks, outputs and messages -- with an
 * environment kept on the device from an earlier run when the
 * configuration's model section and the size and modification time of every
 * data file it names are unchanged (up to four are kept, least recently used
 * evicted), and answers with the exit status and the standard output and
 * error text, which the client prints.  summary.json's environment_seconds
 * is then the look-up.  A client that finds no server fails with
 * "ParaHPOP: no resident environment server answers at <path>: <reason>".
 * After a device error the server answers and stops (returns 1); it also
 * returns 1 when another server answers at the path or it cannot listen.
 * The command line: parahpop_gpu --serve SOCKET, parahpop_gpu --stop SOCKET. */
int phop_resident_serve(const char* socket_path, const char* backend);
/* Asks the server at `socket_path` to stop; 0 when it acknowledged. */
int phop_resident_stop(const char* socket_path);

/* Loads the configuration file's "model" section and its environment files
 * and makes them resident on `device` (the reference's
 * interface::config::Model + Environment::load + model upload,
 * src/common/driver.cpp:132-135, PH/run.h:5-13).  Relative data paths are
 * resolved against the configuration file's directory. */
int phop_create(const char* config_json_path, int device, phop_context** out);

void phop_destroy(phop_context* ctx);

/* Text of the last failure on `ctx` (or of the last failed phop_create when
 * ctx is NULL).  Valid until the next call on the same context. */
const char* phop_last_error(const phop_context* ctx);

/* Run parameters read from the configuration (run.duration_seconds,
 * execution.integration.initialStepSize / maxNumSteps). */
int phop_run_parameters(const phop_context* ctx, double* duration_s, double* step_s, int64_t* max_steps);

/* Propagates n objects (the reference's device Propagator::run,
 * src/common/engine/paraHPOP/propagators/device/Propagator.h:33-66, with the
 * driver's target conversion, src/common/driver.cpp:97-123).
 *   states: n x 6 row-major; duration_s / step_s: per-object arrays, or NULL
 *   for the configuration's values (the reference accepts only one of each).
 * Outputs: final epochs (n) and states (n x 6).  Fails, like the reference,
 * when an object would need more than the configured maxNumSteps. */
int phop_propagate(phop_context* ctx, int64_t n, const double* epoch_mjd2000_tdb, const double* states,
                   const double* mass_kg, const double* drag_area_m2, const double* srp_area_m2, const double* cd,
                   const double* cr, const double* duration_s, const double* step_s, double* out_epoch_mjd2000_tdb,
                   double* out_states);

/* Same propagation with the state already resident in device memory:
 * d_states_soa is a device array of 6*n doubles (x[n], y[n], z[n], vx[n],
 * vy[n], vz[n]) updated in place; every object shares epoch, duration and
 * step.  Other arrays are host arrays.  No counterpart in the reference
 * (which always copies from host); it lets a caller keep batches in HBM. */
int phop_propagate_device(phop_context* ctx, int64_t n, double* d_states_soa, double epoch_mjd2000_tdb,
                          const double* mass_kg, const double* drag_area_m2, const double* srp_area_m2,
                          const double* cd, const double* cr, double duration_s, double step_s,
                          double* out_epoch_mjd2000_tdb);

/* An uneven batch resident in device memory, advanced in slices (the
 * serving loop's pattern, for callers that keep their objects in HBM):
 * phop_object_times fills, on the host, the per-object time arrays the
 * step kernel works on from epochs (MJD2000 TDB), durations and steps (s)
 * with the reference's fixed-step rules (FixedStep.h:7-28 per object:
 * epochs in TDB seconds past J2000, the first step shortened to the span,
 * the maxNumSteps refusal), as 4*n doubles: current epoch[n], end epoch[n],
 * current step size[n] (0 once the end is reached), nominal step[n].
 * phop_propagate_device_objects then advances every object that has not
 * reached its end by at most max_steps fixed steps, on device arrays:
 * d_states_soa (6*n), d_time (4*n, the layout above, updated in place),
 * d_bc and d_ams as for phop_propagate_device_noalloc; *out_unfinished
 * gets the objects still short of their end.  Slices continue exactly where
 * the previous call stopped: any sequence of calls gives, bit for bit, the
 * results of one phop_propagate call over the whole durations at the same
 * lane count.  No reference counterpart (its driver propagates one batch to
 * the end). */
int phop_object_times(const phop_context* ctx, int64_t n, const double* epoch_mjd2000_tdb, const double* duration_s,
                      const double* step_s, double* out_time);
int phop_propagate_device_objects(phop_context* ctx, int64_t n, double* d_states_soa, double* d_time,
                                  const double* d_bc, const double* d_ams, int64_t max_steps,
                                  int64_t* out_unfinished);

/* Trajectory of a batch that shares one epoch, duration and step: the
 * states (n x 6, km and km/s, host arrays in and out) after every
 * `every`-th fixed step, written by the step kernel as it goes.  out_states
 * holds records x n x 6 doubles and out_epochs records doubles (MJD2000 TDB),
 * records = floor(steps / every) with steps = ceil(duration / step); the
 * last record is the final state when `every` divides the step count.  The
 * reference writes final states only; this is the per-step output a serving
 * or screening caller wants instead of re-propagating to each epoch. */
int phop_propagate_trajectory(phop_context* ctx, int64_t n, double epoch_mjd2000_tdb, const double* states,
                              const double* mass_kg, const double* drag_area_m2, const double* srp_area_m2,
                              const double* cd, const double* cr, double duration_s, double step_s, int64_t every,
                              int64_t max_records, double* out_epochs, double* out_states, int64_t* out_records);

/* Allocation-free form of phop_propagate_device.  No counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc while they
 * propagate: a plug-in inside a host application whose own pool allocator
 * has reserved the GPU's memory, a real-time loop that cannot take the
 * device-wide synchronisation a cudaMalloc or cudaFree may imply, or a
 * service that fixes its memory footprint at start-up.  Scratch comes from
 * one 4 MiB device array built into the library, held on every GPU that
 * loads it until the process exits; the call allocates nothing.  The caller
 * passes device arrays: d_states_soa (6*n doubles, updated in place), d_bc =
 * cd * area / mass and d_ams = cr_eff * area / mass (area in km^2, cr_eff =
 * cr * srp_area / drag_area, n doubles each).  Limits: at most 256 fixed
 * steps per call and a coefficient tile of at most 512 KiB (degree/order 120
 * in FP64); larger requests fail with an error, and so does the context
 * option "split_floor_km" (the split form here has the FP32 tile only).
 * The call is synchronous: it returns when the propagation has finished on
 * the GPU.  All calls share the array (the tile it holds is re-copied when a
 * call needs another context's, lane count's or precision's), so calls
 * whose GPU work overlaps race on it: order them.  The first call on a
 * device resolves the array's address and should come before any stream
 * capture. */
int phop_propagate_device_noalloc(phop_context* ctx, int64_t n, double* d_states_soa, const double* d_bc,
                                  const double* d_ams, double epoch_mjd2000_tdb, double duration_s, double step_s,
                                  double* out_epoch_mjd2000_tdb);

/* Execution options (no reference counterpart; the reference hard-codes its
 * launch shapes):
 *   "lanes"    lanes per object, 0 = autotuned, else 1, 2, 4, 8 or 16
 *   "split"    0 = plain FP64, 1 = split precision (FP32 for geopotential
 *              degrees above "split_fp64_degree", FP64 elsewhere)
 *   "split_fp64_degree"  split precision: degrees n <= this (8 .. 24)
 *              stay FP64; default 20, or 24 for fields above degree 80
 *              (FP32 rounding in the recursion of the strongest terms costs
 *              more final-position error than their FP32 speed gains)
 *   "threads"  threads per CTA (multiple of 32, <= 512); a launch uses at
 *              most what the chosen kernel instantiation accepts (its
 *              maxThreadsPerBlock: 256 at 1 lane, 320 at 2, 384 above) and
 *              what shared memory allows
 *   "ctas_per_sm"  resident CTAs per SM, 0 = from occupancy
 *   "ordered"  1 (default) = hand objects to warps in order of geocentric
 *              radius, 0 = in input order; results are identical either way
 *   "graph"    1 (default) = launch the step as a CUDA graph cached by its
 *              launch parameters (replayed for repeated batches), 0 = plain
 *              launches
 *   "tile_smem"  1 (default) = stage the coefficient tile in shared memory
 *              when it fits, 0 = read it through L1 (more threads per SM)
 *   "pair_sh"  geopotential of lane-group pairs, two objects per lane
 *              (each coefficient loaded from shared memory serves both;
 *              packed FP32 in split precision; at one, two or four lanes
 *              only): -1 (default) = chosen by the autotuner with the lane
 *              count (pinned lanes: pairs up to four lanes), 0 = off, 1 = on
 *   "deep_registers"  thread bound of the step kernel at two and four lanes:
 *              1 = 256 threads a CTA with up to 255 registers a thread, 0 =
 *              320 (two lanes) or 384 (four lanes) threads with up to 168;
 *              -1 (default) = chosen by the autotuner (pinned lanes: 0)
 *   "tile_wait_test"  1 = test of the tile-staging time-out: the staging
 *              barrier is armed but no copy issued, so every CTA's bounded
 *              wait runs out and the CTA reads the tile from global memory
 *              (counted in phop_stats.tile_fallbacks); 0 (default) = off
 *   "split_floor_km"  split precision only: objects closer than this height
 *              (km) above the geopotential's reference radius keep every
 *              harmonic in FP64; 0 = none */
int phop_set_option(phop_context* ctx, const char* key, double value);

/* ---- serving loop (no counterpart in the reference, whose driver propagates
 * one batch per process) ----------------------------------------------------
 * A server keeps a device-resident pool of `capacity` object slots (132 bytes
 * of HBM each: the admission budget) on the context's GPU.  Submitted
 * requests queue until their objects fit the pool and the running batch's
 * compute budget (objects one step of the measured rate covers in
 * `slice_ms`, at least 65,536; a larger request runs alone), then join the running
 * batch: each phop_server_step() call admits what fits, launches the step
 * kernel once over every unfinished object of every admitted request for as
 * many fixed steps as fit `slice_ms`, and retires finished requests (their
 * results wait for phop_server_take).  Requests carry per-object epochs,
 * durations and steps; an object's results are bit-identical whichever other
 * requests share its slices.  The server uses its context exclusively while
 * it exists (no phop_propagate* calls on the same context meanwhile) and the
 * context's options ("lanes", "split", "ordered") at creation; without an
 * explicit "lanes" it uses 2.  Failures of a request (maxNumSteps exceeded)
 * are reported by phop_server_take. */
typedef struct phop_server phop_server;

typedef struct {
    int64_t queued, running;      /* requests waiting / admitted now */
    int64_t done, failed;         /* requests finished / failed since creation */
    int64_t active_objects;       /* unfinished objects in the pool */
    int64_t launches;             /* kernels launched by the server */
    int64_t rounds;               /* phop_server_step calls */
    int64_t object_steps;         /* object-steps of finished requests */
    double busy_ms;               /* step-kernel time, CUDA events */
    int lanes;
} phop_server_stats;

int phop_server_create(phop_context* ctx, int64_t capacity, double slice_ms, phop_server** out);
void phop_server_destroy(phop_server* server);
const char* phop_server_last_error(const phop_server* server);
/* Same arrays and checks as phop_propagate; returns a request id. */
int phop_server_submit(phop_server* server, int64_t n, const double* epoch_mjd2000_tdb, const double* states,
                       const double* mass_kg, const double* drag_area_m2, const double* srp_area_m2, const double* cd,
                       const double* cr, const double* duration_s, const double* step_s, int64_t* request_id);
/* One scheduling round; *finished = requests finished or failed in it. */
int phop_server_step(phop_server* server, int64_t* finished);
/* 0 queued, 1 running, 2 done, 3 failed */
int phop_server_status(const phop_server* server, int64_t request_id, int* state);
/* Results of a finished request (epochs n, states n x 6), its latency from
 * submission to completion and its time in the queue, in ms; forgets the
 * request.  Returns 1 with the request's error for a failed request. */
int phop_server_take(phop_server* server, int64_t request_id, double* out_epoch_mjd2000_tdb, double* out_states,
                     double* latency_ms, double* queue_ms);
int phop_server_get_stats(const phop_server* server, phop_server_stats* out);

typedef struct {
    double kernel_ms;        /* step kernel time of the last call, CUDA events */
    double records_ms;       /* epoch-record kernel time of the last call */
    double total_ms;         /* whole call including host<->device copies */
    int64_t object_steps;    /* sum over objects of RKF78 steps taken */
    int64_t launches;        /* kernels launched by the last call */
    int lanes, ctas, threads, split, shared_grid, tile_in_smem;
    double tune_ms;          /* lane-count autotuner probes of the last call (first batch of a size class) */
    int64_t tile_fallbacks;  /* CTAs whose shared-memory staging of the coefficient tile timed out and that
                                read the tile from global memory instead (results are the same) */
    int pair_sh;             /* the geopotential ran for lane-group pairs (two objects per lane) */
    int deep_registers;      /* the step kernel ran at its deep thread bound (256 threads, <= 255 registers) */
    int registers;           /* registers a thread of the step kernel instantiation used */
} phop_stats;

int phop_last_stats(const phop_context* ctx, phop_stats* out);

/* Measured FMA throughput of `device` in TFLOP/s (2 FLOP per FMA), FP64 and
 * FP32: the roofline denominators for the step kernel, which is bound by the
 * FP64 / FP32 pipes rather than by HBM or the tensor cores.  No reference
 * counterpart (the reference reports no roofline). */
int phop_fma_peak(int device, double* fp64_tflops, double* fp32_tflops);

/* NRLMSISE-00 total mass density (kg/m^3, gtd7d with switch 9 = -1) of n
 * input rows {doy, sec, alt_km, g_lat_deg, g_long_deg, lst_h, f107A, f107,
 * ap, ap_a[0..6]} (16 doubles each, row-major), evaluated on `device` by the
 * step kernel's own per-object model with `lanes` (1, 2, 4 or 8) lanes per
 * row.  A known-answer entry: it replaces the reference's gtd7d
 * (model/atmosphere/detail/Nrlmsise00Model.inl:959-1100) called directly.
 * Returns 0, or nonzero with the message in phop_last_error(NULL). */
int phop_nrlmsise00_density(int device, int64_t n, const double* inputs, int lanes, double* out_rho);

/* Reads a configuration and its environment files on the host, with the
 * validation phop_create applies, and needs no device: a configuration check
 * for machines without a GPU.  The files are read and parsed in parallel,
 * one thread per file (errors are those a sequential load meets first).
 * `digest` (optional) receives a 64-bit FNV-1a digest of everything loaded,
 * `load_ms` (optional) the wall time of the load.  Returns 0, or nonzero with
 * the message in phop_last_error(NULL).  The environment part of the
 * reference's driver start-up (src/common/driver.cpp:132-135). */
int phop_load_environment(const char* config_path, uint64_t* digest, double* load_ms);

#ifdef __cplusplus
}
#endif

#endif /* PARAHPOP_B200_H */
