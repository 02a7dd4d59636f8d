"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (run with
``-m gpu`` on a B200); everything else runs on CPU."""
import hashlib
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_names():
    return sorted(p.stem[len("propagation_"):] for p in GOLD.glob("propagation_*.json"))


def env_hash(d: Path) -> str:
    h = hashlib.sha256()
    for name in ("gravity.tab", "bodies.brie", "earth.brot2", "SW-All.txt", "EOP-All.txt", "constants.json"):
        h.update((Path(d) / name).read_bytes())
    if (Path(d) / "moon.tab").exists():  # the lunar field, where a case has one
        h.update((Path(d) / "moon.tab").read_bytes())
    return h.hexdigest()


class GoldenCase:
    """A reference golden case materialised in a directory: environment files
    regenerated by the seeded generator (and checked against the recorded
    hash), config.json and targets.json."""

    def __init__(self, name: str, directory: Path):
        from parahpop_b200 import synthetic as S
        self.name = name
        self.data = json.loads((GOLD / f"propagation_{name}.json").read_text())
        spec = S.EnvSpec(**{k: v for k, v in self.data["env_spec"].items()
                            if k in S.EnvSpec.__dataclass_fields__})
        self.dir = S.write_environment(directory, spec)
        got = env_hash(self.dir)
        assert got == self.data["env_sha256"], "synthetic environment generator drifted from the golden fixture"
        self.config_path = self.dir / "config.json"
        self.targets_path = self.dir / "targets.json"
        self.config_path.write_text(json.dumps(self.data["config"], indent=1))
        self.targets_path.write_text(json.dumps(self.data["targets"]))
        ref = self.data["reference"]
        import numpy as np
        self.ref_ids = np.array(ref["ids"])
        self.ref_epochs = np.array(ref["epochs"])
        self.ref_states = np.array(ref["states"])
        self.targets = self.data["targets"]


@pytest.fixture
def golden(tmp_path):
    def make(name):
        return GoldenCase(name, tmp_path / name)
    return make
