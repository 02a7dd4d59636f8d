"""B200 parity: the CUDA path (through the C ABI) against the reference's own
outputs (golden fixtures) and against the CPU oracle.

Tolerances: the reference's CPU/GPU acceptance, 1 mm in position and
1e-6 m/s in velocity (example/compare.py:7-8), for the plain FP64 path;
1 cm in position for split precision (FP32 for geopotential degrees n > 8).
"""
import json

import numpy as np
import pytest

from conftest import golden_names
from oracle import oracle as O
from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu

POS_TOL_M = 1e-3
VEL_TOL_M_S = 1e-6
SPLIT_POS_TOL_M = 1e-2


def errors(states, ref):
    dpos = np.linalg.norm(states[:, :3] - ref[:, :3], axis=1) * 1e3
    dvel = np.linalg.norm(states[:, 3:] - ref[:, 3:], axis=1) * 1e3
    return dpos.max(), dvel.max()


@pytest.mark.parametrize("name", golden_names())
def test_matches_reference(golden, name):
    case = golden(name)
    p = api.Propagator(case.config_path)
    ep, st = p.propagate_targets(case.targets)
    dpos, dvel = errors(st, case.ref_states)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)
    assert np.abs(ep - case.ref_epochs).max() * 86400.0 <= 1e-4
    p.close()


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("name", ["full_1h", "batch_33"])
def test_every_lane_split_matches(golden, name, lanes):
    case = golden(name)
    p = api.Propagator(case.config_path, lanes=lanes)
    ep, st = p.propagate_targets(case.targets)
    assert p.stats()["lanes"] == lanes
    dpos, dvel = errors(st, case.ref_states)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)


@pytest.mark.parametrize("lanes,pair,deep", [(1, 1, 0), (2, 1, 0), (2, 0, 1), (2, 1, 1), (4, 0, 1), (4, 1, 1)])
@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("name", ["batch_33", "c3_leo_19h"])
def test_every_launch_shape_matches(golden, name, split, lanes, pair, deep):
    """Lane-group pairs and the deep thread bound (256 threads, up to 255
    registers), pinned one shape at a time, on a shared time grid and on
    per-object epochs: each holds the reference bar (FP64 1 mm / 1e-6 m/s,
    split 1 cm), and the statistics report the shape that ran."""
    case = golden(name)
    p = api.Propagator(case.config_path, lanes=lanes, split=split)
    p.set_option("pair_sh", pair)
    p.set_option("deep_registers", deep)
    ep, st = p.propagate_targets(case.targets)
    s = p.stats()
    assert (s["lanes"], s["pair_sh"], s["deep_registers"]) == (lanes, pair, deep)
    assert s["threads"] <= (256 if deep or lanes == 1 else {2: 320, 4: 384}[lanes])
    assert (s["registers"] > 168) == (deep == 1 or lanes == 1), s["registers"]
    dpos, dvel = errors(st, case.ref_states)
    if split:
        assert dpos <= SPLIT_POS_TOL_M, dpos
    else:
        assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)
    p.close()


def test_option_refusals(golden):
    """Out-of-range execution options are refused with a message naming
    them, and leave the context usable."""
    case = golden("full_600s")
    p = api.Propagator(case.config_path)
    for key, bad in (("deep_registers", 2), ("pair_sh", 3), ("split_fp64_degree", 30), ("split_fp64_degree", 7),
                     ("threads", 48), ("threads", 1024), ("lanes", 3), ("split_floor_km", -1.0)):
        with pytest.raises(api.PhopError) as e:
            p.set_option(key, bad)
        assert key in str(e.value), (key, str(e.value))
    with pytest.raises(api.PhopError) as e:
        p.set_option("split_drag_fp32_km", 500.0)
    assert "Unknown option" in str(e.value)
    ep, st = p.propagate_targets(case.targets)
    dpos, dvel = errors(st, case.ref_states)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S
    p.close()


@pytest.mark.parametrize("name", ["full_1h", "deg120_1h", "c1_full_24h", "c2_deg120_24h"])
def test_split_precision_within_1cm(golden, name):
    case = golden(name)
    p = api.Propagator(case.config_path, split=True)
    ep, st = p.propagate_targets(case.targets)
    assert p.stats()["split"] == 1
    dpos, _ = errors(st, case.ref_states)
    assert dpos <= SPLIT_POS_TOL_M, dpos


def test_mixed_population_matches_oracle(tmp_path):
    """Per-object epochs, durations and steps in one persistent launch."""
    d = S.write_environment(tmp_path)
    pop = S.population_mixed(40, seed=31)
    pop.duration = np.minimum(pop.duration, 6 * 3600.0)
    cfg = S.make_config(d, 3600.0, 60.0, max_steps=10 ** 6)
    (d / "config.json").write_text(json.dumps(cfg))
    tg = pop.targets_json()
    p = api.Propagator(d / "config.json")
    ep, st = p.propagate_targets(tg)
    assert p.stats()["shared_grid"] == 0
    env = O.load_environment(d / "config.json")
    _, oep, ost = O.propagate(env, tg)
    dpos, dvel = errors(st, ost)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)
    np.testing.assert_allclose(ep, oep, rtol=0, atol=1e-4 / 86400.0)


def test_command_line_end_to_end(golden):
    case = golden("full_600s")
    out = case.dir / "cli_out"
    r = api.run_cli(case.config_path, case.targets_path, out)
    assert r.returncode == 0, r.stderr
    lines = (out / "final_states.csv").read_text().splitlines()
    assert lines[0] == "id,epoch_mjd2000_tdb,x_km,y_km,z_km,vx_km_s,vy_km_s,vz_km_s"
    _, ep, st = O.read_final_states(out)
    dpos, dvel = errors(st, case.ref_states)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S
    summary = json.loads((out / "summary.json").read_text())
    assert summary["backend"] == "device" and summary["validation_passed"] is True
    assert set(summary) == {"backend", "targets", "integrator", "initial_step_seconds", "duration_seconds",
                            "environment_seconds", "propagation_seconds", "max_end_epoch_error_seconds",
                            "validation_passed"}
    resolved = json.loads((out / "configuration_resolved.json").read_text())
    assert "run" not in resolved and resolved["execution"]["on"] == "device"
    # refuses to overwrite
    r2 = api.run_cli(case.config_path, case.targets_path, out)
    assert r2.returncode == 1 and "Output exists" in r2.stderr


def test_insufficient_max_steps_is_an_error(golden):
    case = golden("full_600s")
    cfg = json.loads(case.config_path.read_text())
    cfg["execution"]["integration"]["maxNumSteps"] = 5
    p2 = case.dir / "c_short.json"
    p2.write_text(json.dumps(cfg))
    r = api.run_cli(p2, case.targets_path, case.dir / "o_short")
    assert r.returncode == 1
    assert "A target stopped without reaching the requested end of simulation." in r.stderr


def test_device_resident_path_equals_host_path(golden):
    case = golden("full_600s")
    import torch
    p = api.Propagator(case.config_path)
    t = case.targets["targets"]
    st0 = np.array([x["state_km_km_s"] for x in t])
    g = lambda k: np.array([x[k] for x in t])
    ep_h, st_h = p.propagate(g("epoch_mjd2000_tdb"), st0, g("mass_kg"), g("drag_area_m2"), g("srp_area_m2"),
                             g("cd"), g("cr"))
    dev = torch.from_numpy(np.ascontiguousarray(st0.T).reshape(-1).copy()).cuda()
    ep_d = p.propagate_device(dev.data_ptr(), len(t), float(t[0]["epoch_mjd2000_tdb"]), g("mass_kg"),
                              g("drag_area_m2"), g("srp_area_m2"), g("cd"), g("cr"), p.duration, p.step)
    st_d = dev.cpu().numpy().reshape(6, -1).T
    np.testing.assert_array_equal(st_d, st_h)
    assert ep_d == ep_h[0]


def test_central_invariants(golden):
    case = golden("central_1d")
    p = api.Propagator(case.config_path)
    _, st = p.propagate_targets(case.targets)
    s0 = np.array([t["state_km_km_s"] for t in case.targets["targets"]])
    mu = 398600.4415
    e0 = 0.5 * (s0[:, 3:] ** 2).sum(1) - mu / np.linalg.norm(s0[:, :3], axis=1)
    e1 = 0.5 * (st[:, 3:] ** 2).sum(1) - mu / np.linalg.norm(st[:, :3], axis=1)
    h0 = np.linalg.norm(np.cross(s0[:, :3], s0[:, 3:]), axis=1)
    h1 = np.linalg.norm(np.cross(st[:, :3], st[:, 3:]), axis=1)
    assert np.abs((e1 - e0) / e0).max() < 1e-9
    assert np.abs((h1 - h0) / h0).max() < 1e-9


def test_benchmark_size_properties(tmp_path):
    """10^4 objects (the benchmark batch) over 30 min: a seeded sample agrees
    with the oracle, repeated runs are bit-identical, and split precision stays
    within 1 cm of FP64 for every object."""
    d = S.write_environment(tmp_path)
    cfg = S.make_config(d, 1800.0, 60.0, max_steps=10 ** 6)
    (d / "config.json").write_text(json.dumps(cfg))
    pop = S.population_leo(10000, 1)
    args = (pop.epochs, pop.states, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr)
    p = api.Propagator(d / "config.json")
    ep1, st1 = p.propagate(*args)
    ep2, st2 = p.propagate(*args)
    np.testing.assert_array_equal(st1, st2)
    ps = api.Propagator(d / "config.json", split=True)
    _, st3 = ps.propagate(*args)
    assert np.linalg.norm(st3[:, :3] - st1[:, :3], axis=1).max() * 1e3 <= SPLIT_POS_TOL_M
    sample = np.random.default_rng(5).choice(10000, 24, replace=False)
    sub = pop.subset(sample)
    env = O.load_environment(d / "config.json")
    _, _, ost = O.propagate(env, sub.targets_json())
    dpos, dvel = errors(st1[sample], ost)
    assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)


def test_graph_replay_equals_plain_launches(golden):
    """The step launch is cached as a CUDA graph: a replayed graph, a fresh
    capture and plain launches give bit-identical results."""
    case = golden("full_600s")
    plain = api.Propagator(case.config_path, lanes=2)
    plain.set_option("graph", 0)
    graphed = api.Propagator(case.config_path, lanes=2)
    _, ref = plain.propagate_targets(case.targets)
    for _ in range(3):  # capture, then replays
        _, st = graphed.propagate_targets(case.targets)
        np.testing.assert_array_equal(st, ref)
    plain.close()
    graphed.close()


def test_split_floor_keeps_low_objects_in_fp64(tmp_path):
    """With split_floor_km, objects below the floor run the FP64 harmonics
    inside the split kernel: the plain FP64 results to rounding for a batch
    that stays below it (the split kernel's FP64 column part ends at degree
    20 instead of 8, so the sums run in another order), and unchanged split
    results far above it."""
    d = S.write_environment(tmp_path)
    cfg = S.make_config(d, 1800.0, 60.0, max_steps=10 ** 6)
    (d / "config.json").write_text(json.dumps(cfg))
    low = S.population_leo(64, 71, alt=(320.0, 450.0))
    high = S.population_leo(64, 72, alt=(1500.0, 2000.0))
    fp64 = api.Propagator(d / "config.json", lanes=2)
    split = api.Propagator(d / "config.json", lanes=2, split=True)
    split.set_option("split_floor_km", 700.0)
    plain_split = api.Propagator(d / "config.json", lanes=2, split=True)
    for pop, same_as_fp64 in ((low, True), (high, False)):
        args = (pop.epochs, pop.states, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr)
        _, a = fp64.propagate(*args)
        _, b = split.propagate(*args)
        _, c = plain_split.propagate(*args)
        if same_as_fp64:
            np.testing.assert_allclose(b, a, rtol=0, atol=1e-9)  # km, km/s: FP64 rounding only
        else:
            np.testing.assert_array_equal(b, c)
        assert np.linalg.norm(b[:, :3] - a[:, :3], axis=1).max() * 1e3 <= SPLIT_POS_TOL_M
    for p in (fp64, split, plain_split):
        p.close()


C3_GROUPS = ["c3_leo_7d", "c3_leo_19h", "c3_meo_2d", "c3_geo_3d"]


def merged_c3(golden):
    """The C3 groups (each pinned by the reference with its own duration and
    step, as the reference command line requires) as ONE uneven batch with
    per-object epochs, durations and steps; ids renumbered."""
    cases = [golden(n) for n in C3_GROUPS]
    merged, refs, spans = [], [], []
    for c in cases:
        for t, ref in zip(c.targets["targets"], c.ref_states):
            t = dict(t, id=len(merged) + 1)
            t["duration_seconds"] = float(c.data["config"]["run"]["duration_seconds"])
            t["step_seconds"] = float(c.data["config"]["execution"]["integration"]["initialStepSize"])
            merged.append(t)
            refs.append(ref)
            spans.append(c.name)
    return cases, {"targets": merged}, np.array(refs), np.array(spans)


@pytest.mark.parametrize("split", [False, True])
def test_c3_groups_in_one_mixed_batch(golden, split):
    """LEO (30 s, up to 7 days), MEO (120 s) and GEO/GTO (300 s, e to 0.7)
    objects with shortened final steps, in one persistent launch, against
    the reference run of each group: 1 mm / 1e-6 m/s in FP64, 1 cm split."""
    cases, tg, refs, groups = merged_c3(golden)
    p = api.Propagator(cases[0].config_path, split=split)
    ep, st = p.propagate_targets(tg)
    assert p.stats()["shared_grid"] == 0
    dpos = np.linalg.norm(st[:, :3] - refs[:, :3], axis=1) * 1e3
    dvel = np.linalg.norm(st[:, 3:] - refs[:, 3:], axis=1) * 1e3
    worst = {g: float(dpos[groups == g].max()) for g in C3_GROUPS}
    if split:
        # the 1 cm bar holds after 24 h; independent FP32 rounding kicks move
        # an orbit along track by an amount that grows as t^1.5, so longer
        # runs get the bar scaled by (t / 24 h)^1.5
        dur = np.array([t["duration_seconds"] for t in tg["targets"]])
        bar = SPLIT_POS_TOL_M * np.maximum(1.0, dur / 86400.0) ** 1.5
        assert (dpos <= bar).all(), worst
    else:
        assert dpos.max() <= POS_TOL_M and dvel.max() <= VEL_TOL_M_S, (worst, dvel.max())
    for c in cases:
        m = groups == c.name
        np.testing.assert_allclose(ep[m], c.ref_epochs, rtol=0, atol=1e-4 / 86400.0)
    p.close()


def test_sliced_resident_batch_equals_one_call(tmp_path):
    """An uneven batch kept in device memory and advanced in slices of at
    most 37 steps per object (phop_propagate_device_objects) ends bit for bit
    where one phop_propagate call over the whole durations ends."""
    import torch
    d = S.write_environment(tmp_path)
    cfg = S.make_config(d, 3600.0, 60.0, max_steps=10 ** 6)
    (d / "config.json").write_text(json.dumps(cfg))
    pop = S.population_mixed(300, seed=37)
    pop.duration = np.minimum(pop.duration, 5 * 3600.0 + 17.0)
    p = api.Propagator(d / "config.json", lanes=2)
    ep1, st1 = p.propagate(pop.epochs, pop.states, pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr,
                           pop.duration, pop.step)
    n = len(pop)
    times = p.object_times(pop.epochs, pop.duration, pop.step)
    bc, ams = api.Propagator.factors(pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr)
    d_state = torch.from_numpy(np.ascontiguousarray(pop.states.T).reshape(-1).copy()).cuda()
    d_time = torch.from_numpy(times).cuda()
    d_bc, d_ams = torch.from_numpy(bc).cuda(), torch.from_numpy(ams).cuda()
    left, calls = n, 0
    while left:
        left = p.propagate_device_objects(n, d_state.data_ptr(), d_time.data_ptr(), d_bc.data_ptr(),
                                          d_ams.data_ptr(), 37)
        calls += 1
        assert calls < 1000
    assert calls > 5
    st2 = d_state.cpu().numpy().reshape(6, n).T
    np.testing.assert_array_equal(st2, st1)
    t = d_time.cpu().numpy()
    np.testing.assert_array_equal(t[:n], t[n:2 * n])      # every object at its end epoch
    np.testing.assert_array_equal(t[2 * n:3 * n], 0.0)   # and finished
    p.close()


def test_tile_staging_timeout_falls_back_to_global_memory(golden):
    """The bounded wait on the tile's bulk copies: with the test switch the
    barrier is armed but no copy issued, every CTA's wait runs out, the CTAs
    read the tile from global memory (counted, not an error), and the
    results are those of the staged tile."""
    case = golden("full_600s")
    ref = api.Propagator(case.config_path, lanes=2)
    _, st_ref = ref.propagate_targets(case.targets)
    assert ref.stats()["tile_in_smem"] == 1 and ref.stats()["tile_fallbacks"] == 0
    t = api.Propagator(case.config_path, lanes=2)
    t.set_option("tile_wait_test", 1)
    _, st = t.propagate_targets(case.targets)
    s = t.stats()
    assert s["tile_in_smem"] == 1 and s["tile_fallbacks"] == s["ctas"] > 0
    np.testing.assert_array_equal(st, st_ref)
    t.set_option("tile_wait_test", 0)
    _, st2 = t.propagate_targets(case.targets)
    assert t.stats()["tile_fallbacks"] == 0
    np.testing.assert_array_equal(st2, st_ref)
    ref.close()
    t.close()
