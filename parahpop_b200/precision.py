"""Workload runs for the larger benchmark configurations: FP64 against split
precision on one population, with throughput and final-position errors.

    python -m parahpop_b200.precision --objects 100000 --degree 120 --hours 24
    python -m parahpop_b200.precision --mixed --objects 1000000 --hours 24

For each precision the population is propagated once through the C ABI
(``phop_propagate``: host arrays in and out, so per-object epochs, durations
and steps are honoured) after an untimed warm-up on a slice of it; the line
printed gives object-steps/s from the kernel events, the split/FP64 speed-up,
and the split-vs-FP64 final-position error percentiles (the FP64 path itself
is held to the reference by the parity tests).  ``--mixed`` uses the
uneven LEO/MEO/GEO population (per-object epochs over +-10 days, durations
capped at ``--hours``).
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

from . import api, synthetic as S


def _errors_m(a, b):
    return np.linalg.norm(a[:, :3] - b[:, :3], axis=1) * 1e3


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--objects", type=int, default=100000)
    ap.add_argument("--degree", type=int, default=70)
    ap.add_argument("--hours", type=float, default=24.0)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--split-floor-km", type=float, default=None,
                    help="split precision: FP64 harmonics below this height (km); default: the library's")
    ap.add_argument("--split-degree", type=int, default=None,
                    help="split precision: degrees n <= this stay FP64 (default: the library's, 20)")
    ap.add_argument("--no-pair", action="store_true", help="one object per lane in the geopotential")
    args = ap.parse_args(argv)

    work = Path(tempfile.mkdtemp(prefix="phop_precision_"))
    S.write_environment(work, S.EnvSpec(degree=args.degree))
    cfg = S.make_config(work, args.hours * 3600.0, 60.0, max_steps=10 ** 8, degree=args.degree)
    (work / "config.json").write_text(json.dumps(cfg))
    if args.mixed:
        pop = S.population_mixed(args.objects, seed=args.seed)
        pop.duration = np.minimum(pop.duration, args.hours * 3600.0)
    else:
        pop = S.population_leo(args.objects, seed=args.seed, screen_duration=args.hours * 3600.0)
        pop.duration = np.full(len(pop), args.hours * 3600.0)
        pop.step = np.full(len(pop), 60.0)
    n = len(pop)
    arrays = (pop.epochs, pop.states, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr, pop.duration, pop.step)
    res = {}
    for name, split in (("fp64", False), ("split", True)):
        p = api.Propagator(work / "config.json", lanes=args.lanes or None, split=split)
        if split and args.split_floor_km is not None:
            p.set_option("split_floor_km", args.split_floor_km)
        if split and args.split_degree is not None:
            p.set_option("split_fp64_degree", args.split_degree)
        if args.no_pair:
            p.set_option("pair_sh", 0)
        warm = pop.subset(np.arange(min(n, 4096)))
        p.propagate(warm.epochs, warm.states, warm.mass, warm.drag_area, warm.srp_area, warm.cd, warm.cr,
                    np.minimum(warm.duration, 1800.0), warm.step)
        t0 = time.perf_counter()
        ep, st = p.propagate(*arrays)
        wall = time.perf_counter() - t0
        s = p.stats()
        res[name] = {"epochs": ep, "states": st, "kernel_ms": s["kernel_ms"], "records_ms": s["records_ms"],
                     "tune_ms": s["tune_ms"],
                     "total_ms": s["total_ms"], "object_steps": s["object_steps"], "lanes": s["lanes"],
                     "wall_s": wall}
        p.close()
    err = _errors_m(res["split"]["states"], res["fp64"]["states"])
    out = {"workload": ("mixed LEO/MEO/GEO" if args.mixed else "LEO") + f", {n} objects, degree {args.degree}, "
                       f"{args.hours:g} h", "object_steps": int(res["fp64"]["object_steps"]),
           "split_floor_km": args.split_floor_km, "split_degree": args.split_degree,
           "pair": not args.no_pair}
    for name in ("fp64", "split"):
        r = res[name]
        out[name] = {"object_steps_per_s": r["object_steps"] / ((r["kernel_ms"] + r["records_ms"]) * 1e-3),
                     "e2e_object_steps_per_s": r["object_steps"] / (r["total_ms"] * 1e-3),
                     "kernel_ms": r["kernel_ms"], "records_ms": r["records_ms"], "tune_ms": r["tune_ms"],
                     "lanes": r["lanes"]}
    out["split_speedup"] = out["split"]["object_steps_per_s"] / out["fp64"]["object_steps_per_s"]
    out["split_vs_fp64_m"] = {"p50": float(np.percentile(err, 50)), "p90": float(np.percentile(err, 90)),
                              "p99": float(np.percentile(err, 99)), "max": float(err.max()),
                              "worst_object": int(err.argmax())}
    # split-vs-FP64 error by initial geocentric radius (altitude bands, km)
    r0 = np.linalg.norm(pop.states[:, :3], axis=1) - S.R_EARTH
    bands = {}
    for lo, hi in ((0, 400), (400, 600), (600, 1000), (1000, 2000), (2000, 1e9)):
        m = (r0 >= lo) & (r0 < hi)
        if m.any():
            bands[f"{lo:g}-{hi:g}"] = {"objects": int(m.sum()), "p99": float(np.percentile(err[m], 99)),
                                       "max": float(err[m].max())}
    out["split_vs_fp64_by_altitude_km"] = bands
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
