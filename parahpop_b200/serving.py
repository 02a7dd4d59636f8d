"""Request traces for the serving loop and a real-time replay driver.

The trace shape follows the serving benchmark configuration: Poisson arrivals,
request sizes log-uniform in objects, durations log-uniform, half of the
requests on a light force model (central + J2-J6 zonal field) and half on the
full force model (degree/order 70).  ``replay`` submits each request when its
arrival time has passed on the wall clock, drives each server's scheduling
rounds from its own host thread, and reports per force model the offered and served object-steps, the
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
    """Replay `trace` against `servers` ({kind: api.Server}) in real time, one
    host thread per server (their slices overlap on the GPU, each server on
    its own stream): requests are submitted when their arrival time has
    passed (up to `horizon_s`), scheduling rounds run until every request
    finished or `horizon_s + drain_s` elapsed.  Returns per force model the
    completed requests, their object-steps per second of wall time and the
    latency / queueing percentiles."""
    import threading

    t0 = time.perf_counter()
    results = {}

    def worker(kind, srv):
        pending = sorted((r for r in trace if r.kind == kind and r.arrival_s <= horizon_s), key=lambda r: r.arrival_s)
        res = {"latency_ms": [], "queue_ms": [], "object_steps": 0, "requests": 0, "submitted": 0}
        live = {}
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival_s <= now:
                r = pending[i]
                sl = slice(r.offset, r.offset + r.n)
                rid = srv.submit(base.epochs[sl], base.states[sl], base.mass[sl], base.drag_area[sl],
                                 base.srp_area[sl], base.cd[sl], base.cr[sl], r.duration_s, step)
                live[rid] = r
                res["submitted"] += 1
                i += 1
            srv.step()
            st = srv.stats()
            busy = st["queued"] > 0 or st["running"] > 0
            for rid in list(live):
                if srv.status(rid) >= 2:
                    r = live.pop(rid)
                    _, _, lat, q = srv.take(rid)
                    res["latency_ms"].append(lat)
                    res["queue_ms"].append(q)
                    res["object_steps"] += r.n * int(np.ceil(r.duration_s / step))
                    res["requests"] += 1
            now = time.perf_counter() - t0
            if (i >= len(pending) and not live) or now > horizon_s + drain_s:
                break
            if not busy and i < len(pending):
                time.sleep(max(0.0, min(pending[i].arrival_s - now, 0.005)))
        res["unfinished"] = len(live)
        results[kind] = res

    threads = [threading.Thread(target=worker, args=(k, srv)) for k, srv in servers.items()]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    wall = time.perf_counter() - t0
    summary = {"wall_s": wall, "unfinished": sum(r["unfinished"] for r in results.values())}
    for kind, res in results.items():
        lat = np.array(res["latency_ms"]) if res["latency_ms"] else np.array([np.nan])
        q = np.array(res["queue_ms"]) if res["queue_ms"] else np.array([np.nan])
        summary[kind] = {"submitted": res["submitted"], "completed": res["requests"], "unfinished": res["unfinished"],
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


def run_trace(preset="fit", seconds=None, drain=60.0, split=False, slice_ms=20.0, hbm_gb=120.0, seed=4,
              device=0) -> dict:
    """Generate the environments and the trace, serve it on `device` with one
    server per force model, and return the replay summary."""
    import json
    import tempfile
    from pathlib import Path

    from . import api

    cfg = dict(PRESETS[preset])
    if seconds:
        cfg["seconds"] = seconds
    work = Path(tempfile.mkdtemp(prefix="phop_serve_"))
    full_dir = S.write_environment(work / "full", S.EnvSpec(degree=70))
    zonal_dir = S.write_environment(work / "zonal", S.EnvSpec(degree=6, zonal_only=True))
    (full_dir / "config.json").write_text(json.dumps(S.make_config(full_dir, 3600.0, 60.0, max_steps=10 ** 7)))
    (zonal_dir / "config.json").write_text(json.dumps(
        S.make_config(zonal_dir, 3600.0, 60.0, max_steps=10 ** 7, force="sh", degree=6)))
    base = S.population_leo(100000, seed=seed, screen_duration=cfg["dur_max"])
    trace = make_trace(seed=seed, **cfg)
    # 132 bytes of HBM per pool slot; the budget is split between the two
    # servers and capped at the largest population a trace can hold at once
    capacity = int(min(hbm_gb * 1e9 / 132 / 2, 4_000_000))
    props = {"zonal": api.Propagator(zonal_dir / "config.json", device=device, split=split),
             "full": api.Propagator(full_dir / "config.json", device=device, split=split)}
    servers = {k: api.Server(p, capacity, slice_ms) for k, p in props.items()}
    summary = replay(servers, base, trace, cfg["seconds"], drain)
    summary["preset"] = preset
    summary["trace"] = cfg
    summary["requests"] = len(trace)
    summary["offered_object_steps"] = offered_object_steps(trace)
    summary["precision"] = "split" if split else "fp64"
    summary["capacity_objects_per_server"] = capacity
    summary["servers"] = {k: srv.stats() for k, srv in servers.items()}
    for srv in servers.values():
        srv.close()
    for p in props.values():
        p.close()
    return summary


def main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--preset", choices=sorted(PRESETS), default="fit")
    ap.add_argument("--seconds", type=float)
    ap.add_argument("--drain", type=float, default=60.0)
    ap.add_argument("--split", action="store_true")
    ap.add_argument("--slice-ms", type=float, default=20.0)
    ap.add_argument("--hbm-gb", type=float, default=120.0, help="admission budget shared by the two servers")
    ap.add_argument("--seed", type=int, default=4)
    args = ap.parse_args(argv)
    summary = run_trace(args.preset, args.seconds, args.drain, args.split, args.slice_ms, args.hbm_gb, args.seed)
    print(json.dumps(summary))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
