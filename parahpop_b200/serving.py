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
    population: S.Population


def _loguniform(rng, lo, hi, n=None):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def make_trace(seconds=60.0, rate=200.0, size_max=1e5, dur_min=600.0, dur_max=3 * 86400.0, step=60.0, seed=4):
    """Poisson arrivals over `seconds`; sizes log-U(1, size_max); durations
    log-U(dur_min, dur_max); kinds alternate at random 50/50."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        n = max(1, int(_loguniform(rng, 1.0, size_max)))
        dur = float(_loguniform(rng, dur_min, dur_max))
        kind = "zonal" if rng.uniform() < 0.5 else "full"
        pop = S.population_leo(n, seed=seed * 100003 + k, screen_duration=dur)
        pop.duration = np.full(n, dur)
        pop.step = np.full(n, step)
        out.append(TraceRequest(t, kind, pop))
        k += 1
    return out


def offered_object_steps(trace) -> dict:
    out = {}
    for r in trace:
        steps = int(np.ceil(r.population.duration[0] / r.population.step[0]))
        out[r.kind] = out.get(r.kind, 0) + len(r.population) * steps
    return out


def replay(servers: dict, trace, horizon_s: float | None = None) -> dict:
    """Replay `trace` against `servers` ({kind: api.Server}) in real time.
    Stops taking new arrivals after `horizon_s` (default: the trace length)
    and returns once every submitted request has finished."""
    t0 = time.perf_counter()
    pending = sorted(trace, key=lambda r: r.arrival_s)
    horizon = horizon_s if horizon_s is not None else (pending[-1].arrival_s if pending else 0.0)
    live = {}
    results = {k: {"latency_ms": [], "queue_ms": [], "object_steps": 0, "requests": 0} for k in servers}
    i = 0
    while True:
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i].arrival_s <= min(now, horizon):
            r = pending[i]
            p = r.population
            rid = servers[r.kind].submit(p.epochs, p.states, p.mass, p.drag_area, p.srp_area, p.cd, p.cr,
                                         p.duration, p.step)
            live[(r.kind, rid)] = r
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
                res["object_steps"] += len(r.population) * int(np.ceil(r.population.duration[0] / r.population.step[0]))
                res["requests"] += 1
        done_arrivals = i >= len(pending) or pending[i].arrival_s > horizon
        if done_arrivals and not busy and not live:
            break
        if not busy and i < len(pending):
            time.sleep(max(0.0, min(pending[i].arrival_s - (time.perf_counter() - t0), 0.01)))
    wall = time.perf_counter() - t0
    summary = {"wall_s": wall}
    for kind, res in results.items():
        lat = np.array(res["latency_ms"]) if res["latency_ms"] else np.array([np.nan])
        q = np.array(res["queue_ms"]) if res["queue_ms"] else np.array([np.nan])
        summary[kind] = {"requests": res["requests"], "object_steps": res["object_steps"],
                         "served_object_steps_per_s": res["object_steps"] / wall,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "queue_p50_ms": float(np.percentile(q, 50)), "queue_p99_ms": float(np.percentile(q, 99))}
    return summary
