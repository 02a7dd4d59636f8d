"""Benchmark: batched fixed-step RKF78 full-force propagation on B200.

Default workload: the uneven population of the headline configuration --
10^6 objects per GPU, 70 % LEO (30 s step), 20 % MEO (120 s), 10 % GEO/GTO
(300 s, e up to 0.7), per-object epochs over +-10 days and durations
log-uniform 1 h - 7 d, full force model at degree/order 70 (tides folded
into the low degrees, NRLMSISE-00 drag, SRP with Earth shadow, Sun / Moon /
Jupiter third body, Schwarzschild term).  The population is resident in HBM
and advanced in slices: one benchmark step is one persistent launch that
advances every unfinished object by up to S fixed steps of its own size
(phop_propagate_device_objects), so the K timed steps cover each object's
first K*S steps.  Both precision forms are timed; the headline value is the
fastest form whose measured final-position error stays within 1 cm (the
`parity` block: against the reference CPU backend's own outputs, and split
precision against FP64 over whole 24 h runs).  Metric: object-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3|c1|c2] [--impl reference]

`--workload c1` is the 10^4-object LEO batch (24 h at 60 s, one shared time
grid), `c2` the 10^5-object degree-120 batch.  Under torchrun each rank
propagates its own population (weak scaling; objects are independent, no
data-path collective) and rank 0 prints one JSON line with the whole-job
throughput (max time over ranks).
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
SPLIT_TOL_M = 1e-2
FP64_TOL_M = 1e-3


def sh_terms(degree: int) -> float:
    return (degree + 1) * (degree + 2) / 2.0


def sh_flops_per_object_step(degree: int) -> float:
    return 13.0 * SH_FLOP_PER_TERM * sh_terms(degree)


# DRAM bytes (read + write) per object-step of the step kernel, from ncu
# captures (profiles/): the state is read once and written once per launch
# (~100 B per object); the rest is local memory written back from L2 and the
# epoch-record grid.  c3: the split form's kernel at two lanes with lane-group
# pairs and the 256-thread bound, 10^5 objects x 24 steps (8.77 + 5.82 GB over
# 2,391,620 object-steps); the other workloads have no capture of the current
# kernel (null).
NCU_BYTES_PER_OBJECT_STEP = {"c3": (8.769621e9 + 5.815049e9) / 2_391_620, "c1": None, "c2": None}


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


# ---------------------------------------------------------------------------
# the reference CPU backend (bounded samples)
# ---------------------------------------------------------------------------
def _reference_env():
    env = dict(os.environ, OMP_DYNAMIC="FALSE", OMP_WAIT_POLICY="PASSIVE")
    try:
        import ctypes
        ctypes.CDLL("libcuda.so.1")
    except OSError:
        shim = ROOT / "oracle" / "_ref" / "libnodrv_shim.so"
        if shim.exists():
            env["LD_PRELOAD"] = str(shim)
    return env


def run_reference_cli(env_dir: Path, pop, duration: float, step: float, threads: int, degree: int = 70,
                      backend: str = "cpu") -> dict:
    """One run of a reference backend (oracle/_ref/bin/parahpop_cpu or
    parahpop_gpu, built from the reference sources): its command line takes
    one duration and one step for all targets.  `seconds` is the
    `propagation_seconds` of its summary.json (model and cache set-up,
    transfers, graph construction and replay; not the environment load)."""
    from parahpop_b200 import synthetic as S
    binary = ROOT / "oracle" / "_ref" / "bin" / f"parahpop_{backend}"
    if not binary.exists():
        return {"unavailable": f"{binary.relative_to(ROOT)} not built"}
    cfg = S.make_config(env_dir, duration, step, max_steps=10 ** 6, threads=threads, degree=degree)
    tag = f"{len(pop)}_{int(duration)}_{int(step)}"
    cfgp, tgp = env_dir / f"{backend}_config_{tag}.json", env_dir / f"{backend}_targets_{tag}.json"
    cfgp.write_text(json.dumps(cfg))
    tg = pop.targets_json()
    for t in tg["targets"]:  # one duration and step per run
        t.pop("duration_seconds", None)
        t.pop("step_seconds", None)
    tgp.write_text(json.dumps(tg))
    out = Path(tempfile.mkdtemp(prefix=f"{backend}_ref_", dir=env_dir))
    shutil.rmtree(out)
    env = _reference_env() if backend == "cpu" else dict(os.environ)
    r = subprocess.run([str(binary), str(cfgp), str(tgp), str(out)], cwd=env_dir, env=env,
                       capture_output=True, text=True)
    if r.returncode != 0:
        return {"unavailable": f"reference {backend.upper()} run failed: "
                               + (r.stderr.strip().splitlines() or ["?"])[-1]}
    summ = json.loads((out / "summary.json").read_text())
    shutil.rmtree(out, ignore_errors=True)
    steps = int(np.ceil(duration / step))
    return {"seconds": summ["propagation_seconds"], "object_steps": len(pop) * steps}


def c3_cpu_sample(threads: int):
    """A bounded C3 sample for the reference CPU backend: per orbit class a
    group of objects (their own epochs) sharing one duration and the class's
    step, as the reference command line requires."""
    from parahpop_b200 import synthetic as S
    pop = S.population_mixed(20000, seed=91)
    groups = []
    for step, count in ((30.0, 48 * threads), (120.0, 16 * threads), (300.0, 8 * threads)):
        idx = np.flatnonzero(pop.step == step)[:count]
        groups.append((pop.subset(idx), 3600.0, step))
    return groups


def time_reference_c3(work: Path, threads: int) -> dict:
    groups = c3_cpu_sample(threads)
    secs, obj = 0.0, 0
    for pop, dur, step in groups:
        r = run_reference_cli(work, pop, dur, step, threads)
        if "unavailable" in r:
            return r
        secs += r["seconds"]
        obj += r["object_steps"]
    sample = ", ".join(f"{len(p)} objects at {s:g} s" for p, _, s in groups)
    return {"value": obj / secs, "seconds": secs, "object_steps": obj,
            "sample": f"C3 population sample, 1 h per orbit class ({sample}), one reference run per (step, "
                      f"duration) group, {secs:.2f} s on {threads} threads"}


def time_reference_c1(work: Path, threads: int) -> dict:
    from parahpop_b200 import synthetic as S
    n = min(10000, 64 * threads)
    pop = S.population_leo(n, 11)
    r = run_reference_cli(work, pop, 3600.0, 60.0, threads)
    if "unavailable" in r:
        return r
    return {"value": r["object_steps"] / r["seconds"], "seconds": r["seconds"], "object_steps": r["object_steps"],
            "sample": f"{n} objects x 1 h (60 steps) of the 10^4-object LEO workload, {r['seconds']:.2f} s on "
                      f"{threads} threads"}


def time_reference_gpu(work: Path, workload: str) -> dict:
    """The reference's own GPU backend (oracle/_ref/bin/parahpop_gpu, built
    from the reference sources for sm_100a) on the same GPU: for C1 the whole
    10^4-object population for 1 h, for C3 each orbit class of a 10^5-object
    draw of the population for 1 h, one run per (step, duration) group as its
    command line requires.  Throughput = object-steps / propagation_seconds
    (its summary.json), the timing scope of the reference's
    scripts/benchmark_gpu.py."""
    from parahpop_b200 import synthetic as S
    if workload == "c3":
        pop = S.population_mixed(100000, seed=91)
        groups = [(pop.subset(np.flatnonzero(pop.step == st)), 3600.0, st) for st in (30.0, 120.0, 300.0)]
    else:
        groups = [(S.population_leo(10000 if workload == "c1" else 100000, 11), 3600.0, 60.0)]
    secs, obj = 0.0, 0
    for pop, dur, step in groups:
        r = run_reference_cli(work, pop, dur, step, 1, degree=120 if workload == "c2" else 70, backend="gpu")
        if "unavailable" in r:
            return r
        secs += r["seconds"]
        obj += r["object_steps"]
    sample = ", ".join(f"{len(p)} objects at {s:g} s" for p, _, s in groups)
    return {"value": obj / secs, "unit": "object-steps/s", "seconds": secs, "object_steps": obj,
            "kind": "reference GPU backend (parahpop_gpu built from the reference sources for sm_100a)",
            "sample": f"1 h per group ({sample}), propagation_seconds summed: {secs:.2f} s"}


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from parahpop_b200 import synthetic as S
    threads = os.cpu_count() or 1
    work = Path(tempfile.mkdtemp(prefix="phop_ref_bench_"))
    S.write_environment(work, S.EnvSpec(degree=70))
    timer = time_reference_c3 if args.workload == "c3" else time_reference_c1
    timer(work, threads) if args.warmup > 0 else None  # page cache and binary warm
    vals, res = [], None
    for _ in range(args.steps):
        res = timer(work, threads)
        if "unavailable" in res:
            print(json.dumps({"impl": "reference", "unavailable": res["unavailable"]}))
            return 0
        vals.append(res)
    secs = sum(r["seconds"] for r in vals)
    value = sum(r["object_steps"] for r in vals) / secs
    wl = WORKLOAD_NAMES[args.workload] + " (bounded CPU sample)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "object-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl},
            "cpu_baseline": {"value": value, "unit": "object-steps/s", "cores": threads, "kind": "reference",
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": "object-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    shutil.rmtree(work, ignore_errors=True)
    return 0


WORKLOAD_NAMES = {
    "c3": "uneven population: 10^6 objects per GPU (70% LEO at 30 s, 20% MEO at 120 s, 10% GEO/GTO at 300 s), "
          "per-object epochs +-10 d and durations log-U(1 h, 7 d), full force degree/order 70",
    "c1": "10^4 LEO objects per GPU, full force, degree/order 70, 24 h at 60 s",
    "c2": "10^5 LEO objects per GPU, full force, degree/order 120, 24 h at 60 s",
}


# ---------------------------------------------------------------------------
# parity: final-position errors of both forms
# ---------------------------------------------------------------------------
def _pct(err_km):
    e = np.asarray(err_km) * 1e6
    return {"p50_mm": float(np.percentile(e, 50)), "p99_mm": float(np.percentile(e, 99)), "max_mm": float(e.max()),
            "objects": int(len(e))}


def parity_block(work: Path, device: int, split_degree: int | None) -> dict:
    """Errors against the reference CPU backend's own final states (the
    committed golden fixtures made by it: C1 24 h and the C3 orbit-class
    groups merged into one uneven launch), and split precision against FP64
    over whole 24 h runs (the C1 configuration in full, and 10^5 objects of
    the C3 population with durations capped at 24 h)."""
    from parahpop_b200 import api, synthetic as S
    gold = ROOT / "tests" / "golden"
    out = {}

    def forms(cfg_path, fn):
        res = {}
        for name, split in (("fp64", False), ("split", True)):
            p = api.Propagator(cfg_path, device=device, split=split)
            if split and split_degree is not None:
                p.set_option("split_fp64_degree", split_degree)
            res[name] = fn(p)
            p.close()
        return res

    # against the reference's outputs
    cases = {}
    for name in ("c1_full_24h", "c3_leo_7d", "c3_leo_19h", "c3_meo_2d", "c3_geo_3d"):
        cases[name] = json.loads((gold / f"propagation_{name}.json").read_text())
    d = S.write_environment(work / "parity", S.EnvSpec(**cases["c1_full_24h"]["env_spec"]))
    cfgp = d / "config.json"
    cfgp.write_text(json.dumps(cases["c1_full_24h"]["config"]))
    targets, refs = [], []
    for name, c in cases.items():
        dur = c["config"]["run"]["duration_seconds"]
        step = c["config"]["execution"]["integration"]["initialStepSize"]
        for t, r in zip(c["targets"]["targets"], c["reference"]["states"]):
            t = dict(t, id=len(targets) + 1, duration_seconds=dur, step_seconds=step)
            targets.append(t)
            refs.append(r)
    refs = np.array(refs)
    dur = np.array([t["duration_seconds"] for t in targets])
    res = forms(cfgp, lambda p: p.propagate_targets({"targets": targets})[1])
    err = {k: np.linalg.norm(res[k][:, :3] - refs[:, :3], axis=1) for k in res}
    day = dur <= 86400.0
    out["vs_reference"] = {
        "sample": f"{len(targets)} objects: C1 24 h ({len(cases['c1_full_24h']['targets']['targets'])} LEO incl. "
                  "300-400 km) and the C3 orbit classes (LEO 7 d and 19 h, MEO 2 d, GEO/GTO 3 d) in one uneven "
                  "launch; reference = parahpop_cpu final states",
        "fp64": _pct(err["fp64"]),
        "split_up_to_24h": _pct(err["split"][day]),
        "split_beyond_24h": _pct(err["split"][~day])}
    # 1 cm after 24 h; beyond, FP32 rounding kicks grow the along-track error as t^1.5
    split_bar_km = SPLIT_TOL_M * 1e-3 * np.maximum(1.0, dur / 86400.0) ** 1.5
    # split against FP64 over whole 24 h runs
    c1 = S.population_leo(10000, 1)
    res = forms(cfgp, lambda p: p.propagate(c1.epochs, c1.states, c1.mass, c1.drag_area, c1.srp_area, c1.cd, c1.cr,
                                            duration=86400.0, step=60.0)[1])
    out["split_vs_fp64_c1_24h"] = _pct(np.linalg.norm(res["split"][:, :3] - res["fp64"][:, :3], axis=1))
    c3 = S.population_mixed(100000, seed=5)
    c3.duration = np.minimum(c3.duration, 86400.0)
    res = forms(cfgp, lambda p: p.propagate(c3.epochs, c3.states, c3.mass, c3.drag_area, c3.srp_area, c3.cd, c3.cr,
                                            c3.duration, c3.step)[1])
    out["split_vs_fp64_c3_24h"] = _pct(np.linalg.norm(res["split"][:, :3] - res["fp64"][:, :3], axis=1))
    out["split_vs_fp64_c3_24h"]["sample"] = "10^5 objects of the C3 population, durations capped at 24 h"
    out["split_within_1cm"] = bool((err["split"] <= split_bar_km).all()
                                   and out["split_vs_fp64_c1_24h"]["max_mm"] <= SPLIT_TOL_M * 1e3
                                   and out["split_vs_fp64_c3_24h"]["max_mm"] <= SPLIT_TOL_M * 1e3)
    out["split_bar"] = "1 cm after 24 h (runs beyond 24 h: 1 cm x (t / 24 h)^1.5)"
    out["fp64_within_1mm"] = bool(out["vs_reference"]["fp64"]["max_mm"] <= FP64_TOL_M * 1e3)
    return out


# ---------------------------------------------------------------------------
# the timed runs
# ---------------------------------------------------------------------------
class Timer:
    """CUDA events on the launching (default) stream around each step."""

    def __init__(self):
        import torch
        self.torch = torch
        self.ms = []

    def __enter__(self):
        self.a = self.torch.cuda.Event(enable_timing=True)
        self.b = self.torch.cuda.Event(enable_timing=True)
        self.torch.cuda.synchronize()
        self.a.record()
        return self

    def __exit__(self, *exc):
        self.b.record()
        self.b.synchronize()
        self.ms.append(self.a.elapsed_time(self.b))


def c3_run(prop, pop, slices: int, warmup: int, steps_per_slice: int, flush, e2e: bool) -> dict:
    """W warm-up slices on a scratch copy, then K timed slices: device-
    resident (value), or with every slice's inputs copied from pinned host
    memory and its results read back inside the timed region (e2e)."""
    import torch
    n = len(pop)
    times0 = prop.object_times(pop.epochs, pop.duration, pop.step)
    bc, ams = prop.factors(pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr)
    soa0 = np.ascontiguousarray(pop.states.T).reshape(-1)
    h_state = torch.from_numpy(soa0.copy()).pin_memory()
    h_time = torch.from_numpy(times0.copy()).pin_memory()
    h_bc = torch.from_numpy(bc).pin_memory()
    h_ams = torch.from_numpy(ams).pin_memory()
    d_state = h_state.cuda()
    d_time = h_time.cuda()
    d_bc = h_bc.cuda()
    d_ams = h_ams.cuda()
    # warm-up on a scratch copy (first slices of the population: the lane
    # autotuner's probes run here)
    s_state, s_time = d_state.clone(), d_time.clone()
    for _ in range(warmup):
        prop.propagate_device_objects(n, s_state.data_ptr(), s_time.data_ptr(), d_bc.data_ptr(), d_ams.data_ptr(),
                                      steps_per_slice)
    del s_state, s_time
    torch.cuda.synchronize()
    timer = Timer()
    kernel_ms = records_ms = 0.0
    obj_steps = launches = 0
    lanes = None
    for k in range(slices):
        flush.fill_(k & 0xFF)  # evict L2 between timed steps
        with timer:
            if e2e:
                d_state.copy_(h_state, non_blocking=True)
                d_time.copy_(h_time, non_blocking=True)
                d_bc.copy_(h_bc, non_blocking=True)
                d_ams.copy_(h_ams, non_blocking=True)
            prop.propagate_device_objects(n, d_state.data_ptr(), d_time.data_ptr(), d_bc.data_ptr(),
                                          d_ams.data_ptr(), steps_per_slice)
            if e2e:
                h_state.copy_(d_state, non_blocking=True)
                h_time.copy_(d_time, non_blocking=True)
        st = prop.stats()
        kernel_ms += st["kernel_ms"]
        records_ms += st["records_ms"]
        obj_steps += st["object_steps"]
        launches += st["launches"]
        lanes = st["lanes"]
        pairs = st["pair_sh"]
    return {"ms": timer.ms, "kernel_ms": kernel_ms, "records_ms": records_ms, "object_steps": obj_steps,
            "launches": launches, "lanes": lanes, "pairs": pairs,
            "state": d_state.cpu().numpy().reshape(6, n).T.copy(),
            "h2d_bytes": n * (6 + 4 + 2) * 8, "d2h_bytes": n * (6 + 4) * 8}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c3", "c1", "c2"])
    ap.add_argument("--objects", type=int, default=0, help="objects per GPU (default: the workload's)")
    ap.add_argument("--slice-steps", type=int, default=24, help="c3: fixed steps per object per benchmark step")
    ap.add_argument("--hours", type=float, default=24.0, help="c1/c2: span covered by the K timed steps")
    ap.add_argument("--split-degree", type=int, default=None, help="split precision: FP64 up to this degree")
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--pair-sh", type=int, default=-1, choices=[-1, 0, 1],
                    help="geopotential of lane-group pairs: -1 autotuned (pinned lanes: on up to 4 lanes)")
    ap.add_argument("--deep-registers", type=int, default=-1, choices=[-1, 0, 1],
                    help="thread bound at 2 and 4 lanes: 1 deep (256 threads, 255 registers), 0 wide, -1 autotuned")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity leg")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip timing the reference's GPU backend")
    ap.add_argument("--serving-seconds", type=float, default=8.0,
                    help="arrival window of the serving trace (C4 shape) per precision form (0: skip)")
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

    degree = 120 if args.workload == "c2" else 70
    work = Path(tempfile.mkdtemp(prefix=f"phop_bench_{rank}_"))
    S.write_environment(work, S.EnvSpec(degree=degree))
    K, W = args.steps, args.warmup
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    fp64_peak, fp32_peak = api.fma_peak(local)

    def sync_barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    runs = {}
    clocks = ClockSampler(local)
    if args.workload == "c3":
        n_obj = args.objects or 1_000_000
        cfg = S.make_config(work, 3600.0, 60.0, max_steps=10 ** 7, degree=degree)
        (work / "config.json").write_text(json.dumps(cfg))
        pop = S.population_mixed(n_obj, seed=3 + rank)
        for name, split in (("fp64", False), ("split", True)):
            prop = api.Propagator(work / "config.json", device=local, lanes=args.lanes or None, split=split)
            if split and args.split_degree is not None:
                prop.set_option("split_fp64_degree", args.split_degree)
            prop.set_option("pair_sh", args.pair_sh)
            prop.set_option("deep_registers", args.deep_registers)
            sync_barrier()
            if name == "fp64":
                clocks.start()
            r = c3_run(prop, pop, K, W, args.slice_steps, flush, e2e=False)
            sync_barrier()
            r["e2e"] = c3_run(prop, pop, K, 0, args.slice_steps, flush, e2e=True)
            if name == "split":
                r["clocks"] = clocks.stop()
            prop.close()
            runs[name] = r
    else:
        n_obj = args.objects or (10000 if args.workload == "c1" else 100000)
        step_s = 60.0
        span = args.hours * 3600.0 / K
        cfg = S.make_config(work, span, step_s, max_steps=10 ** 7, degree=degree)
        (work / "config.json").write_text(json.dumps(cfg))
        pop = S.population_leo(n_obj, seed=1 + rank)
        for name, split in (("fp64", False), ("split", True)):
            prop = api.Propagator(work / "config.json", device=local, lanes=args.lanes or None, split=split)
            if split and args.split_degree is not None:
                prop.set_option("split_fp64_degree", args.split_degree)
            prop.set_option("pair_sh", args.pair_sh)
            prop.set_option("deep_registers", args.deep_registers)
            soa = np.ascontiguousarray(pop.states.T).reshape(-1)
            d_state = torch.from_numpy(soa.copy()).cuda()
            scratch = d_state.clone()
            for _ in range(W):
                scratch.copy_(d_state)
                prop.propagate_device(scratch.data_ptr(), pop.__len__(), float(pop.epochs[0]), pop.mass,
                                      pop.drag_area, pop.srp_area, pop.cd, pop.cr, span, step_s)
            sync_barrier()
            if name == "fp64":
                clocks.start()
            timer = Timer()
            r = {"kernel_ms": 0.0, "records_ms": 0.0, "object_steps": 0, "launches": 0}
            epoch = float(pop.epochs[0])
            for k in range(K):
                flush.fill_(k & 0xFF)
                with timer:
                    epoch = prop.propagate_device(d_state.data_ptr(), len(pop), epoch, pop.mass, pop.drag_area,
                                                  pop.srp_area, pop.cd, pop.cr, span, step_s)
                st = prop.stats()
                for key in ("kernel_ms", "records_ms", "object_steps", "launches"):
                    r[key] += st[key]
                r["lanes"] = st["lanes"]
                r["pairs"] = st["pair_sh"]
            sync_barrier()
            r["ms"] = timer.ms
            r["state"] = d_state.cpu().numpy().reshape(6, -1).T.copy()
            # end to end through phop_propagate with host arrays
            states, epochs = pop.states.copy(), pop.epochs.copy()
            e2e_ms, e2e_steps = 0.0, 0
            for k in range(K):
                flush.fill_(k & 0xFF)
                with Timer() as t:
                    epochs, states = prop.propagate(epochs, states, pop.mass, pop.drag_area, pop.srp_area, pop.cd,
                                                    pop.cr, duration=span, step=step_s)
                e2e_ms += t.ms[0]
                e2e_steps += prop.stats()["object_steps"]
            r["e2e"] = {"ms": [e2e_ms / K] * K, "object_steps": e2e_steps, "h2d_bytes": len(pop) * 14 * 8,
                        "d2h_bytes": len(pop) * 7 * 8}
            if name == "split":
                r["clocks"] = clocks.stop()
            prop.close()
            runs[name] = r

    # whole-job throughput per form (max time over ranks)
    forms = {}
    for name, r in runs.items():
        t_ms = max_over_ranks(sum(r["ms"]))
        e_ms = max_over_ranks(sum(r["e2e"]["ms"]))
        forms[name] = {"value": r["object_steps"] * ws / (t_ms * 1e-3), "ms_per_step": t_ms / K,
                       "e2e_value": r["e2e"]["object_steps"] * ws / (e_ms * 1e-3),
                       "kernel_ms": r["kernel_ms"], "records_ms": r["records_ms"], "lanes": r["lanes"],
                       "objects_per_lane_in_geopotential": 2 if r["pairs"] else 1,
                       "object_steps_per_gpu": r["object_steps"], "launches": r["launches"]}
    prefix_diff = np.linalg.norm(runs["split"]["state"][:, :3] - runs["fp64"]["state"][:, :3], axis=1)

    parity = None
    cpu = None
    ref_gpu = None
    serving = None
    if rank == 0:
        if not args.no_parity:
            parity = parity_block(work, local, args.split_degree)
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            r = time_reference_c3(work, threads) if args.workload == "c3" else time_reference_c1(work, threads)
            if "unavailable" in r:
                cpu = {"value": None, "unit": "object-steps/s", "cores": threads, "kind": "reference",
                       "sample": r["unavailable"]}
            else:
                cpu = {"value": r["value"], "unit": "object-steps/s", "cores": threads, "kind": "reference",
                       "sample": r["sample"]}
        if not args.no_reference_gpu:
            ref_gpu = time_reference_gpu(work, args.workload)
        if args.serving_seconds > 0:
            from parahpop_b200 import serving as SV
            serving = {}
            for name, split in (("fp64", False), ("split", True)):
                summ = SV.run_trace("full", seconds=args.serving_seconds, drain=2.0 * args.serving_seconds,
                                    split=split, device=local)
                blk = {"trace": f"{summ['requests']} requests, Poisson {summ['trace']['rate']:g}/s over "
                                f"{summ['trace']['seconds']:g} s (then {2 * args.serving_seconds:g} s of drain), "
                                f"sizes log-U(1, {summ['trace']['size_max']:g}), durations "
                                f"log-U({summ['trace']['dur_min']:g}, {summ['trace']['dur_max']:g}) s, half "
                                "central+J2-J6, half full force degree 70, HBM budget 120 GB",
                       "offered_object_steps": summ["offered_object_steps"], "unfinished": summ["unfinished"]}
                for kind in ("zonal", "full"):
                    k = summ[kind]
                    blk[kind] = {"p50_ms": k["p50_ms"], "p99_ms": k["p99_ms"], "queue_p99_ms": k["queue_p99_ms"],
                                 "completed": k["completed"], "submitted": k["submitted"],
                                 "served_object_steps_per_s": k["served_object_steps_per_s"]}
                serving[name] = blk

    if rank == 0:
        ok_split = parity is None or parity["split_within_1cm"]
        head = "split" if ok_split and forms["split"]["value"] > forms["fp64"]["value"] else "fp64"
        h = forms[head]
        r = runs[head]
        flops = sh_flops_per_object_step(degree) * r["object_steps"]
        achieved = flops / (r["kernel_ms"] * 1e-3) * 1e-12
        if head == "split":
            low = args.split_degree or (24 if degree > 80 else 20)  # the library's default by field degree
            f64 = 13.0 * SH_FLOP_PER_TERM * sh_terms(low)
            f32 = sh_flops_per_object_step(degree) - f64
            peak = sh_flops_per_object_step(degree) / (f64 / fp64_peak + f32 / fp32_peak)
            peak_note = (f"FMA peaks measured on this GPU (phop_fma_peak: FP64 {fp64_peak:.1f}, FP32 "
                         f"{fp32_peak:.1f} TFLOP/s), weighted by the split's FP64 (n <= {low}) and FP32 terms")
        else:
            peak = fp64_peak
            peak_note = "measured FP64 FMA throughput (phop_fma_peak) on this GPU"
        per_os = NCU_BYTES_PER_OBJECT_STEP.get(args.workload)
        steps_per_launch = r["object_steps"] / K
        line = {
            "metric": METRIC, "value": h["value"], "unit": "object-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": h["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if head == "split" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAMES[args.workload] + (
                f"; one step = one launch advancing every unfinished object by up to {args.slice_steps} fixed "
                f"steps (the K timed steps cover each object's first {K * args.slice_steps} steps)"
                if args.workload == "c3" else f"; {K} steps of {args.hours / K:.2f} h"),
                       "objects_per_gpu": n_obj, "degree": degree, "precision": head,
                       "split_fp64_degree": args.split_degree or (24 if degree > 80 else 20), "lanes": h["lanes"],
                       "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"object sharding x{ws}, no collective"},
            "forms": {"fp64": forms["fp64"], "split": forms["split"],
                      "split_speedup": forms["split"]["value"] / forms["fp64"]["value"],
                      "split_vs_fp64_after_timed_steps": _pct(prefix_diff)},
            "roofline": {"bound": "fp64+fp32" if head == "split" else "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None,
                         "traffic": per_os * steps_per_launch if per_os else None,
                         "traffic_note": "DRAM read+write bytes per launch: ncu capture of the split kernel at two "
                                         "lanes, lane-group pairs, 256-thread bound (6.1 KB per object-step: "
                                         "local-memory write-back and epoch-record reads) times the object-steps of "
                                         "one timed launch" if per_os else None,
                         "peak_source": peak_note,
                         "numerator": f"29 FLOP x (N+1)(N+2)/2 SH terms x 13 stages per object-step, N = {degree}"},
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "e2e": {"value": h["e2e_value"], "unit": "object-steps/s", "h2d_bytes_per_step": r["e2e"]["h2d_bytes"],
                    "d2h_bytes_per_step": r["e2e"]["d2h_bytes"]},
            "parity": parity,
            "serving": serving,
            "gpu_launches": h["launches"],
            "clocks": runs["split"].get("clocks"),
            "fp64_peak_tflops": fp64_peak, "fp32_peak_tflops": fp32_peak,
        }
        print(json.dumps(line))
    shutil.rmtree(work, ignore_errors=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
