"""Serving loop (phop_server_*): continuous batching of requests with their own
epochs, durations and steps.

* A request's results are bit-identical whether it is served alone or joins a
  running mix of other requests part-way through.
* Served results agree with the CPU oracle within the reference's CPU/GPU
  acceptance (1 mm, 1e-6 m/s; example/compare.py:7-8).
* Requests beyond the configured maxNumSteps fail with the driver's message,
  requests larger than the pool are refused, and a pool smaller than the
  offered load queues requests until slots free up.
"""
import json

import numpy as np
import pytest

from oracle import oracle as O
from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu

POS_TOL_M = 1e-3
VEL_TOL_M_S = 1e-6


def _env(tmp_path, max_steps=10 ** 6):
    d = S.write_environment(tmp_path)
    cfg = S.make_config(d, 3600.0, 60.0, max_steps=max_steps)
    (d / "config.json").write_text(json.dumps(cfg))
    return d


def _mixed(n, seed, cap_s):
    p = S.population_mixed(n, seed=seed)
    p.duration = np.minimum(p.duration, cap_s)
    return p


def _serve(prop, requests, capacity=4096, stagger=0):
    """Submit `requests` (targets dicts), `stagger` rounds apart; returns the
    results by position and the server statistics."""
    srv = api.Server(prop, capacity, slice_ms=5.0)
    ids = []
    for tg in requests:
        ids.append(srv.submit_targets(tg))
        for _ in range(stagger):
            srv.step()
    srv.run_until_idle()
    out = [srv.take(i) for i in ids]
    st = srv.stats()
    srv.close()
    return out, st


def test_results_identical_alone_and_in_mix(tmp_path):
    d = _env(tmp_path)
    a = _mixed(48, 41, 3 * 3600.0).targets_json()
    b = _mixed(300, 42, 6 * 3600.0).targets_json()
    c = S.population_leo(200, 43).targets_json()
    prop = api.Propagator(d / "config.json")
    (alone,), _ = _serve(prop, [a])
    mixed, st = _serve(prop, [b, a, c], stagger=3)
    np.testing.assert_array_equal(mixed[1][0], alone[0])
    np.testing.assert_array_equal(mixed[1][1], alone[1])
    assert st["done"] == 3 and st["failed"] == 0 and st["lanes"] == 2
    # and against the CPU oracle
    env = O.load_environment(d / "config.json")
    _, oep, ost = O.propagate(env, a)
    dpos = np.linalg.norm(alone[1][:, :3] - ost[:, :3], axis=1).max() * 1e3
    dvel = np.linalg.norm(alone[1][:, 3:] - ost[:, 3:], axis=1).max() * 1e3
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)
    np.testing.assert_allclose(alone[0], oep, rtol=0, atol=1e-4 / 86400.0)
    prop.close()


def test_queueing_when_pool_is_full(tmp_path):
    d = _env(tmp_path)
    prop = api.Propagator(d / "config.json")
    reqs = [S.population_leo(100, 50 + k).targets_json() for k in range(5)]
    for tg in reqs:
        for t in tg["targets"]:
            t["duration_seconds"] = 1200.0
    srv = api.Server(prop, 250, slice_ms=5.0)
    ids = [srv.submit_targets(tg) for tg in reqs]
    srv.step()
    st = srv.stats()
    assert st["running"] == 2 and st["queued"] == 3  # 250 slots hold two requests of 100
    srv.run_until_idle()
    out = [srv.take(i) for i in ids]
    assert srv.stats()["done"] == 5
    srv.close()
    ref = api.Propagator(d / "config.json", lanes=2)
    for tg, (ep, stt, lat, q) in zip(reqs, out):
        assert lat >= q >= 0.0
        _, st2 = ref.propagate_targets(tg)
        # the uniform path evaluates epoch records exactly instead of
        # interpolating them: equal within the parity tolerance
        assert np.linalg.norm(stt[:, :3] - st2[:, :3], axis=1).max() * 1e3 <= POS_TOL_M
    ref.close()
    prop.close()


def test_step_limit_and_capacity_errors(tmp_path):
    d = _env(tmp_path, max_steps=10)
    prop = api.Propagator(d / "config.json")
    srv = api.Server(prop, 64)
    tg = S.population_leo(8, 60).targets_json()
    for t in tg["targets"]:
        t["duration_seconds"] = 1800.0  # 30 steps > maxNumSteps = 10
    rid = srv.submit_targets(tg)
    srv.run_until_idle()
    assert srv.status(rid) == api.Server.FAILED
    with pytest.raises(api.PhopError, match="A target stopped without reaching the requested end of simulation."):
        srv.take(rid)
    with pytest.raises(api.PhopError, match="exceeds the server capacity"):
        srv.submit_targets(S.population_leo(65, 61).targets_json())
    srv.close()
    prop.close()
