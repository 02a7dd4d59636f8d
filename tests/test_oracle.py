"""The CPU oracle against the reference's own outputs (golden fixtures made
by the reference CPU backend and model sources built from the reference
tree, see tests/golden/make_golden.py)."""
import json

import numpy as np
import pytest

from conftest import GOLD, golden_names
from oracle import oracle as O


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_propagation(golden, name):
    case = golden(name)
    env = O.load_environment(case.config_path)
    ids, ep, st = O.propagate(env, case.targets, threads=4)
    assert list(ids) == list(case.ref_ids)
    # reference acceptance (example/compare.py:7-8): 1 mm, 1e-6 m/s; the
    # restatement is ten times inside it up to a day.  Beyond a day (the
    # week-long LEO run) rounding differences grow along track to a few
    # 1e-4 m, and the bar is the acceptance itself.
    dpos = np.linalg.norm(st[:, :3] - case.ref_states[:, :3], axis=1) * 1e3
    dvel = np.linalg.norm(st[:, 3:] - case.ref_states[:, 3:], axis=1) * 1e3
    longest = max([float(t.get("duration_seconds", 0.0)) for t in case.targets["targets"]]
                  + [float(case.data["config"]["run"]["duration_seconds"])])
    pos_tol, vel_tol = (1e-4, 1e-7) if longest <= 86400.0 else (1e-3, 1e-6)
    assert dpos.max() < pos_tol, dpos.max()
    assert dvel.max() < vel_tol, dvel.max()
    assert np.abs(ep - case.ref_epochs).max() * 86400 < 1e-9


def test_nrlmsise00_known_answers():
    kat = json.loads((GOLD / "nrlmsise00_kat.json").read_text())
    for v, rho in zip(kat["inputs"], kat["rho_kg_m3"]):
        got = O.nrl_density(int(v[0]), v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9:16])
        assert got == pytest.approx(rho, rel=1e-13, abs=0.0), (v, got, rho)


def test_tides_known_answers():
    import ctypes as C
    kat = json.loads((GOLD / "tides_kat.json").read_text())
    lib = O.lib()
    D = C.POINTER(C.c_double)
    lib.oracle_tides.argtypes = [D] * 5 + [C.c_double] * 5 + [D] * 7
    for v, out in zip(kat["inputs"], kat["outputs"]):
        a = np.array(v, dtype=np.float64)
        bufs = [np.zeros(49) for _ in range(4)] + [np.zeros(3) for _ in range(3)]
        p = lambda x: x.ctypes.data_as(D)
        lib.oracle_tides(p(a[0:3]), p(a[3:6]), p(a[6:9]), p(a[9:12]), p(a[12:21]), a[21], a[22], a[23], a[24], a[25],
                         *[p(b) for b in bufs])
        for got, key in zip(bufs[:4], ("solidC", "solidS", "oceanC", "oceanS")):
            np.testing.assert_allclose(got, out[key], rtol=1e-12, atol=1e-20)
        for got, key in zip(bufs[4:], ("solid", "ocean", "rel")):
            np.testing.assert_allclose(got, out[key], rtol=1e-10, atol=1e-22)


def test_central_invariants_over_a_day(golden):
    """Central gravity conserves energy and angular momentum (validate.py:90-105)."""
    case = golden("central_1d")
    mu = 398600.4415
    s0 = np.array([t["state_km_km_s"] for t in case.targets["targets"]])
    s1 = case.ref_states
    for s in (s1,):
        e0 = 0.5 * (s0[:, 3:] ** 2).sum(1) - mu / np.linalg.norm(s0[:, :3], axis=1)
        e1 = 0.5 * (s[:, 3:] ** 2).sum(1) - mu / np.linalg.norm(s[:, :3], axis=1)
        h0 = np.linalg.norm(np.cross(s0[:, :3], s0[:, 3:]), axis=1)
        h1 = np.linalg.norm(np.cross(s[:, :3], s[:, 3:]), axis=1)
        assert np.abs((e1 - e0) / e0).max() < 1e-9
        assert np.abs((h1 - h0) / h0).max() < 1e-9
