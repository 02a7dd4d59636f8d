"""Synthetic environment generator: determinism, formats, populations."""
import json

import numpy as np

from conftest import GOLD, env_hash
from oracle.oracle import cbor_loads
from parahpop_b200 import synthetic as S


def test_environment_is_deterministic(tmp_path):
    a = S.write_environment(tmp_path / "a")
    b = S.write_environment(tmp_path / "b")
    assert env_hash(a) == env_hash(b)
    gold = json.loads((GOLD / "propagation_full_600s.json").read_text())
    assert env_hash(a) == gold["env_sha256"]


def test_cbor_round_trip():
    obj = {"layout": 1, "core": [{"metadata": {"a": -3, "b": 2.5, "c": "x" * 30}, "data": [1.0, -2.0, 3e300]}]}
    assert cbor_loads(S.cbor_dumps(obj)) == obj


def test_brie_units_cover_the_window(tmp_path):
    d = S.write_environment(tmp_path)
    units = cbor_loads((d / "bodies.brie").read_bytes())["core"]
    assert {u["metadata"]["target"] for u in units} == {10, 399, 301, 5}
    for u in units:
        m = u["metadata"]
        assert len(u["data"]) == 1 + m["nintervals"] + 3 * (m["pdeg"] + 1) * m["nintervals"]
        assert m["startEpoch"] <= S.mjd2000_to_et(4025.0) and m["finalEpoch"] >= S.mjd2000_to_et(4052.0)


def test_population_shapes_and_decay_screen():
    p = S.population_leo(2000, 1)
    r = np.linalg.norm(p.states[:, :3], axis=1)
    assert (r > S.R_EARTH + 200).all() and (r < S.R_EARTH + 2100).all()
    assert S.decay_km(r, 0 * r, 2.2, p.drag_area, p.mass, 86400.0).max() <= 25.0
    m = S.population_mixed(5000, 3)
    assert m.duration.min() >= 3600.0 and m.duration.max() <= 7 * 86400.0
    assert set(np.unique(m.step)) == {30.0, 120.0, 300.0}
    assert np.abs(m.epochs - S.EPOCH0).max() <= 10.0


def test_kepler_circular_speed():
    st = S.kepler_to_state(7000.0, 0.0, 0.5, 0.1, 0.2, 0.3)
    assert abs(np.linalg.norm(st[3:]) - np.sqrt(S.MU_ELEMENTS / 7000.0)) < 1e-12
