"""Host logic of the device tide model (parahpop_b200/csrc/tide_field.cuh,
written from the IERS Conventions 2010 ch. 6): its solid (zero-tide) and
FES2004 ocean coefficient sets against the reference's own
HpopCorrections.h on the known-answer inputs (tests/golden/tides_kat.json,
made by oracle/_ref/ref_kat).  Compiled for the host with nvcc (no GPU
needed); on the device the same pieces run one warp per epoch and are held
to the reference by the propagation goldens."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not Path(NVCC).exists(), reason="nvcc not available")
def test_tide_sets_match_reference_known_answers(tmp_path):
    exe = tmp_path / "tide_check"
    subprocess.run([NVCC, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", str(ROOT / "parahpop_b200" / "csrc"),
                    str(ROOT / "tests" / "tide_check.cu"), "-o", str(exe)], check=True)
    kat = json.loads((ROOT / "tests" / "golden" / "tides_kat.json").read_text())
    stdin = "\n".join(" ".join(repr(float(x)) for x in v) for v in kat["inputs"]) + "\n"
    out = subprocess.run([str(exe)], input=stdin, check=True, capture_output=True, text=True).stdout
    got = [json.loads(line) for line in out.splitlines()]
    assert len(got) == len(kat["outputs"])
    for g, ref in zip(got, kat["outputs"]):
        for key in ("solidC", "solidS", "oceanC", "oceanS"):
            a, b = np.array(g[key]), np.array(ref[key])
            # relative to the set's largest coefficient: the sets mix
            # corrections of 1e-8 (degree 2) with 1e-13 (degree 6)
            scale = np.abs(b).max()
            assert np.abs(a - b).max() <= 1e-12 * scale, (key, np.abs(a - b).max(), scale)
