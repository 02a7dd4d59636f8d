"""The device NRLMSISE-00 (the step kernel's per-object model, with its
epoch-block coefficient rows and lane split) against the reference's own
gtd7d outputs on the known-answer grid (0-1000 km, all branches: below
72.5 km, the mesosphere nodes, the low-altitude species corrections and the
thermosphere)."""
import json
from pathlib import Path

import numpy as np
import pytest

from parahpop_b200 import api

pytestmark = pytest.mark.gpu

KAT = Path(__file__).resolve().parent / "golden" / "nrlmsise00_kat.json"


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
def test_device_density_matches_reference(lanes):
    kat = json.loads(KAT.read_text())
    inputs = np.array(kat["inputs"], dtype=np.float64)
    ref = np.array(kat["rho_kg_m3"])
    got = api.nrlmsise00_density(inputs, lanes=lanes)
    rel = np.abs(got - ref) / np.abs(ref)
    assert np.all(np.isfinite(got))
    assert rel.max() < 1e-12, (rel.max(), inputs[rel.argmax()][:6])


def test_rejects_bad_lane_count():
    with pytest.raises(api.PhopError, match="lanes"):
        api.nrlmsise00_density(np.zeros((1, 16)), lanes=3)
