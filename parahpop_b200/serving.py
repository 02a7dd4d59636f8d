"""Request traces for the serving loop and a real-time replay driver.

The trace shape follows the serving benchmark configuration: Poisson arrivals,
request sizes log-uniform in objects, durations log-uniform, half of the
requests on a light force model (central + J2-J6 zonal field) and half on the
full force model (degree/order 70).  ``replay`` submits each request when its
arrival time has passed on the wall clock, drives the servers' scheduling
rounds, and reports per force model the offered and served object-steps, the
request latency percentiles (submission to completion) and the queueing
delay.  The full-size trace (200 req/s, up to 10^5 objects and 3 days per
request) offers ~10^11 object-steps per minute, far beyond one GPU; a
scaled trace keeps the distributions' shapes with smaller bounds.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import synthetic as S


@dataclass
class TraceRequest:
    arrival_s: float
    kind: str            # "zonal" | "full"
    offset: int          # first object in the base population
    n: int
    duration_s: float


def _loguniform(rng, lo, hi, n=None):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def make_trace(seconds=60.0, rate=200.0, size_max=1e5, dur_min=600.0, dur_max=3 * 86400.0, base_size=100000,
               seed=4):
    """Poisson arrivals over `seconds`; sizes log-U(1, size_max) (contiguous
    slices of a base population of `base_size` objects); durations
    log-U(dur_min, dur_max); each request on the zonal or the full force
    model with probability 1/2."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        n = int(min(base_size, max(1, int(_loguniform(rng, 1.0, size_max)))))
        dur = float(_loguniform(rng, dur_min, dur_max))
        kind = "zonal" if rng.uniform() < 0.5 else "full"
        out.append(TraceRequest(t, kind, int(rng.integers(0, base_size - n + 1)), n, dur))
    return out


def offered_object_steps(trace, step=60.0) -> dict:
    out = {}
    for r in trace:
        out[r.kind] = out.get(r.kind, 0) + r.n * int(np.ceil(r.duration_s / step))
    return out


def replay(servers: dict, base: S.Population, trace, horizon_s: float, drain_s: float, step=60.0) -> dict:
    """Replay `trace` against `servers` ({kind: api.Server}) in real time:
    requests are submitted when their arrival time has passed (up to
    `horizon_s`), scheduling rounds run until every request finished or
    `horizon_s + drain_s` elapsed.  Returns per force model the completed
    requests, served object-steps/s and the latency / queueing percentiles."""
    t0 = time.perf_counter()
    pending = sorted((r for r in trace if r.arrival_s <= horizon_s), key=lambda r: r.arrival_s)
    live = {}
    results = {k: {"latency_ms": [], "queue_ms": [], "object_steps": 0, "requests": 0, "submitted": 0}
               for k in servers}
    i = 0
    while True:
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i].arrival_s <= now:
            r = pending[i]
            sl = slice(r.offset, r.offset + r.n)
            rid = servers[r.kind].submit(base.epochs[sl], base.states[sl], base.mass[sl], base.drag_area[sl],
                                         base.srp_area[sl], base.cd[sl], base.cr[sl], r.duration_s, step)
            live[(r.kind, rid)] = r
            results[r.kind]["submitted"] += 1
            i += 1
        busy = False
        for kind, srv in servers.items():
            srv.step()
            st = srv.stats()
            busy |= st["queued"] > 0 or st["running"] > 0
        for key in list(live):
            kind, rid = key
            if servers[kind].status(rid) >= 2:
                r = live.pop(key)
                _, _, lat, q = servers[kind].take(rid)
                res = results[kind]
                res["latency_ms"].append(lat)
                res["queue_ms"].append(q)
                res["object_steps"] += r.n * int(np.ceil(r.duration_s / step))
                res["requests"] += 1
        now = time.perf_counter() - t0
        if i >= len(pending) and not live:
            break
        if now > horizon_s + drain_s:
            break
        if not busy and i < len(pending):
            time.sleep(max(0.0, min(pending[i].arrival_s - now, 0.005)))
    wall = time.perf_counter() - t0
    summary = {"wall_s": wall, "unfinished": len(live)}
    for kind, res in results.items():
        lat = np.array(res["latency_ms"]) if res["latency_ms"] else np.array([np.nan])
        q = np.array(res["queue_ms"]) if res["queue_ms"] else np.array([np.nan])
        summary[kind] = {"submitted": res["submitted"], "completed": res["requests"],
                         "object_steps": res["object_steps"],
                         "served_object_steps_per_s": res["object_steps"] / wall,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "queue_p50_ms": float(np.percentile(q, 50)), "queue_p99_ms": float(np.percentile(q, 99))}
    return summary


PRESETS = {
    # the serving configuration's distributions at full size (overloads one GPU)
    "full": dict(seconds=60.0, rate=200.0, size_max=1e5, dur_min=600.0, dur_max=3 * 86400.0),
    # the same shapes with bounds one GPU serves without a growing queue
    "fit": dict(seconds=60.0, rate=20.0, size_max=1e4, dur_min=600.0, dur_max=7200.0),
}


def main(argv=None):
    import argparse
    import json
    import tempfile
    from pathlib import Path

    from . import api

    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--preset", choices=sorted(PRESETS), default="fit")
    ap.add_argument("--seconds", type=float)
    ap.add_argument("--drain", type=float, default=60.0)
    ap.add_argument("--split", action="store_true")
    ap.add_argument("--slice-ms", type=float, default=20.0)
    ap.add_argument("--hbm-gb", type=float, default=120.0, help="admission budget shared by the two servers")
    ap.add_argument("--seed", type=int, default=4)
    args = ap.parse_args(argv)
    cfg = dict(PRESETS[args.preset])
    if args.seconds:
        cfg["seconds"] = args.seconds
    work = Path(tempfile.mkdtemp(prefix="phop_serve_"))
    full_dir = S.write_environment(work / "full", S.EnvSpec(degree=70))
    zonal_dir = S.write_environment(work / "zonal", S.EnvSpec(degree=6, zonal_only=True))
    (full_dir / "config.json").write_text(json.dumps(S.make_config(full_dir, 3600.0, 60.0, max_steps=10 ** 7)))
    (zonal_dir / "config.json").write_text(json.dumps(
        S.make_config(zonal_dir, 3600.0, 60.0, max_steps=10 ** 7, force="sh", degree=6)))
    base = S.population_leo(100000, seed=args.seed, screen_duration=cfg["dur_max"])
    trace = make_trace(seed=args.seed, **cfg)
    # 132 bytes of HBM per pool slot; the budget is split between the two
    # servers and capped at the largest population a trace can hold at once
    capacity = int(min(args.hbm_gb * 1e9 / 132 / 2, 4_000_000))
    props = {"zonal": api.Propagator(zonal_dir / "config.json", split=args.split),
             "full": api.Propagator(full_dir / "config.json", split=args.split)}
    servers = {k: api.Server(p, capacity, args.slice_ms) for k, p in props.items()}
    summary = replay(servers, base, trace, cfg["seconds"], args.drain)
    summary["preset"] = args.preset
    summary["trace"] = cfg
    summary["requests"] = len(trace)
    summary["offered_object_steps"] = offered_object_steps(trace)
    summary["precision"] = "split" if args.split else "fp64"
    summary["capacity_objects_per_server"] = capacity
    summary["servers"] = {k: srv.stats() for k, srv in servers.items()}
    print(json.dumps(summary))
    for srv in servers.values():
        srv.close()
    for p in props.values():
        p.close()
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
