"""Benchmark: batched fixed-step RKF78 full-force propagation on B200.

Workload (the benchmark's headline configuration): 10^4 LEO objects, full
force model (degree/order 70 geopotential with solid + ocean tides folded in,
NRLMSISE-00 drag, SRP with Earth shadow, Sun / Moon / Jupiter third body,
Schwarzschild term), 24 h at a 60 s step, FP64 (plain) unless --split.  One
benchmark step propagates the batch over 24h / K (K = --steps), continuing
from the previous step's states, so K timed steps cover the full day; the W
warm-up steps propagate a scratch copy.  Metric: object-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--split] [--impl reference]

Under torchrun each rank propagates its own 10^4 objects (weak scaling; the
objects are independent, there is no data-path collective) and rank 0 prints
one JSON line with the whole-job throughput (max time over ranks).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "object-steps/s full-force at ≤1 cm vs FP64 oracle; p50/p99 request latency"
SH_FLOP_PER_TERM = 29  # algorithmic FLOPs per (n, m) term of the SH recursion


def sh_flops_per_object_step(degree: int) -> float:
    return 13.0 * SH_FLOP_PER_TERM * (degree + 1) * (degree + 2) / 2.0


# DRAM bytes (read + write) of one step-kernel launch over 10^4 objects and 5
# steps at eight lanes, from an ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum); a longer launch reads one more 896-byte epoch record
# per added stage.
NCU_BYTES_5_STEPS_1E4 = 1_570_560 + 1_846_016
RECORD_BYTES = 896


def launch_traffic_bytes(objects: int, steps: int) -> float:
    per_object = (NCU_BYTES_5_STEPS_1E4 - 13 * 5 * RECORD_BYTES) / 1e4
    return per_object * objects + 13 * steps * RECORD_BYTES


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference(n_objects: int, threads: int, env_dir: Path, duration: float, step: float, seed: int = 11) -> dict:
    """Time the reference CPU backend (oracle/_ref/bin/parahpop_cpu, built
    from the reference sources) on a bounded sample of the workload."""
    from parahpop_b200 import synthetic as S
    binary = ROOT / "oracle" / "_ref" / "bin" / "parahpop_cpu"
    if not binary.exists():
        return {"unavailable": f"{binary} not built"}
    pop = S.population_leo(n_objects, seed)
    cfg = S.make_config(env_dir, duration, step, max_steps=100000, threads=threads)
    cfgp = env_dir / f"cpu_config_{n_objects}.json"
    tgp = env_dir / f"cpu_targets_{n_objects}.json"
    cfgp.write_text(json.dumps(cfg))
    tgp.write_text(json.dumps(pop.targets_json()))
    out = Path(tempfile.mkdtemp(prefix="cpu_ref_", dir=env_dir))
    shutil.rmtree(out)
    env = dict(os.environ, OMP_DYNAMIC="FALSE", OMP_WAIT_POLICY="PASSIVE")
    try:
        import ctypes
        ctypes.CDLL("libcuda.so.1")
    except OSError:
        shim = ROOT / "oracle" / "_ref" / "libnodrv_shim.so"
        if shim.exists():
            env["LD_PRELOAD"] = str(shim)
    r = subprocess.run([str(binary), str(cfgp), str(tgp), str(out)], cwd=env_dir, env=env, capture_output=True,
                       text=True)
    if r.returncode != 0:
        return {"unavailable": "reference CPU run failed: " + (r.stderr.strip().splitlines() or ["?"])[-1]}
    summ = json.loads((out / "summary.json").read_text())
    steps = int(np.ceil(duration / step))
    return {"value": n_objects * steps / summ["propagation_seconds"], "seconds": summ["propagation_seconds"],
            "object_steps": n_objects * steps}


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from parahpop_b200 import synthetic as S
    threads = os.cpu_count() or 1
    work = Path(tempfile.mkdtemp(prefix="phop_ref_bench_"))
    S.write_environment(work, S.EnvSpec(degree=70))
    duration, step = 3600.0, 60.0
    n = min(10000, 64 * threads)
    cpu_reference(min(n, 2 * threads), threads, work, 600.0, step)  # warm the page cache
    times = []
    res = None
    for _ in range(args.steps):
        res = cpu_reference(n, threads, work, duration, step)
        if "unavailable" in res:
            print(json.dumps({"impl": "reference", "unavailable": res["unavailable"]}))
            return 0
        times.append(res["seconds"])
    obj_steps = res["object_steps"]
    value = obj_steps * len(times) / sum(times)
    sample = f"{n} objects x 1 h (60 steps) of the 10^4-object full-force LEO workload, degree 70, per step"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "object-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "10^4 LEO full force, degree/order 70, 24 h at 60 s (bounded CPU sample)",
                       "objects": n, "degree": 70},
            "cpu_baseline": {"value": value, "unit": "object-steps/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "object-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    shutil.rmtree(work, ignore_errors=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--split", action="store_true", help="split precision (FP32 for n > 8)")
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--objects", type=int, default=10000)
    ap.add_argument("--hours", type=float, default=24.0, help="propagated span covered by the K timed steps")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--serving-seconds", type=float, default=15.0,
                    help="length of the request trace replayed for the p50/p99 latency leg (0: skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    from parahpop_b200 import api, synthetic as S

    work = Path(tempfile.mkdtemp(prefix=f"phop_bench_{rank}_"))
    S.write_environment(work, S.EnvSpec(degree=70))
    K, W = args.steps, args.warmup
    step_s = 60.0
    span = args.hours * 3600.0 / K
    cfg = S.make_config(work, span, step_s, max_steps=10 ** 7)
    (work / "config.json").write_text(json.dumps(cfg))
    pop = S.population_leo(args.objects, seed=1 + rank)
    n = len(pop)
    prop = api.Propagator(work / "config.json", device=local, lanes=args.lanes or None, split=args.split)
    fp64_peak, fp32_peak = api.fma_peak(local)

    def sync_barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    # ---- device-resident throughput (value) --------------------------------
    soa = np.ascontiguousarray(pop.states.T).reshape(-1)
    d_state = torch.from_numpy(soa.copy()).cuda()
    d_scratch = torch.from_numpy(soa.copy()).cuda()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    epoch0 = float(pop.epochs[0])
    for _ in range(W):
        d_scratch.copy_(d_state)
        torch.cuda.synchronize()
        prop.propagate_device(d_scratch.data_ptr(), n, epoch0, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr,
                              span, step_s)
    clocks = ClockSampler(local)
    kernel_ms = 0.0
    launches = 0
    obj_steps = 0
    step_ms = []
    sync_barrier()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    epoch = epoch0
    total_ms = 0.0
    for k in range(K):
        flush.fill_(k & 0xFF)  # evict L2 between timed steps
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        epoch = prop.propagate_device(d_state.data_ptr(), n, epoch, pop.mass, pop.drag_area, pop.srp_area, pop.cd,
                                      pop.cr, span, step_s)
        torch.cuda.synchronize()
        st = prop.stats()
        ms = st["records_ms"] + st["kernel_ms"]
        step_ms.append(ms)
        total_ms += ms
        kernel_ms += st["kernel_ms"]
        launches += st["launches"]
        obj_steps += st["object_steps"]
    sync_barrier()
    clk = clocks.stop()
    final_dev = d_state.cpu().numpy().reshape(6, n).T.copy()
    max_ms = total_ms
    if ws > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        max_ms = float(t.item())
    value = obj_steps * ws / (max_ms * 1e-3)
    flops = sh_flops_per_object_step(70) * obj_steps
    achieved = flops / (kernel_ms * 1e-3) * 1e-12
    peak = fp32_peak if False else fp64_peak

    # ---- end to end through the C ABI with host buffers (e2e) ----------------
    states = pop.states.copy()
    epochs = pop.epochs.copy()
    e2e_ms = 0.0
    h2d = d2h = 0
    sync_barrier()
    for k in range(K):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        epochs, states = prop.propagate(epochs, states, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr,
                                        duration=span, step=step_s)
        e2e_ms += prop.stats()["total_ms"]
        h2d = n * (6 + 1 + 5 + 2) * 8
        d2h = n * (6 + 1) * 8
    sync_barrier()
    e2e_max = e2e_ms
    if ws > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_max = float(t.item())
    e2e_value = obj_steps * ws / (e2e_max * 1e-3)
    consistent = float(np.abs(states - final_dev).max())

    # ---- CPU baseline (reference CPU backend, bounded sample) ------------------
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        nc = min(10000, 64 * threads)
        r = cpu_reference(nc, threads, work, 3600.0, step_s)
        if "unavailable" in r:
            cpu = {"value": None, "unit": "object-steps/s", "cores": threads, "kind": "reference",
                   "sample": r["unavailable"]}
        else:
            cpu = {"value": r["value"], "unit": "object-steps/s", "cores": threads, "kind": "reference",
                   "sample": f"{nc} objects x 1 h (60 steps), same force model and field, "
                             f"{r['seconds']:.2f} s on {threads} threads"}
    # ---- serving latency (request trace, continuous batching) ----------------
    serving = None
    if rank == 0 and args.serving_seconds > 0:
        from parahpop_b200 import serving as SV
        summ = SV.run_trace("fit", seconds=args.serving_seconds, drain=60.0, split=args.split, device=local)
        serving = {"trace": f"{summ['requests']} requests, Poisson {summ['trace']['rate']:g}/s over "
                            f"{summ['trace']['seconds']:g} s, sizes log-U(1, {summ['trace']['size_max']:g}), "
                            f"durations log-U({summ['trace']['dur_min']:g}, {summ['trace']['dur_max']:g}) s, "
                            "half central+J2-J6, half full force degree 70",
                   "unfinished": summ["unfinished"]}
        for kind in ("zonal", "full"):
            k = summ[kind]
            serving[kind] = {"p50_ms": k["p50_ms"], "p99_ms": k["p99_ms"], "queue_p99_ms": k["queue_p99_ms"],
                             "completed": k["completed"],
                             "served_object_steps_per_s": k["served_object_steps_per_s"]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "object-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.split else "f64", "data": "synthetic",
            "config": {"workload": "10^4 LEO objects per GPU, full force, degree/order 70, 24 h at 60 s "
                                   f"({K} steps of {span / 3600:.1f} h)",
                       "objects_per_gpu": n, "degree": 70, "precision": "split" if args.split else "fp64",
                       "lanes": prop.stats()["lanes"], "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"object sharding x{ws}, no collective"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak > 0 else None,
                         "traffic": launch_traffic_bytes(n, int(round(span / step_s))),
                         "traffic_note": "DRAM bytes per launch: ncu capture of a 5-step launch of the same "
                                         "10^4 objects at eight lanes (3.417 MB read+write) plus 896 B per further stage "
                                         "record",
                         "peak_source": "measured FP64 FMA throughput (phop_fma_peak) on this GPU",
                         "numerator": "29 FLOP x (N+1)(N+2)/2 SH terms x 13 stages per object-step, N = 70"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "object-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "serving": serving,
            "gpu_launches": launches,
            "clocks": clk,
            "fp32_peak_tflops": fp32_peak,
            "device_vs_host_path_max_abs_diff": consistent,
        }
        print(json.dumps(line))
    prop.close()
    shutil.rmtree(work, ignore_errors=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
