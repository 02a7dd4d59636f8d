"""Host logic of the device NRLMSISE-00: the per-(day, ap slot) globe7
coefficient rows (nrl_fast.cuh, nrlGlobeRows) reproduce the term-by-term
globe7 of the straight restatement on random inputs.  Compiled for the host
with nvcc (no GPU needed); the device side is held to the reference's gtd7d
by tests/test_gpu_nrlmsise00.py."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not Path(NVCC).exists(), reason="nvcc not available")
def test_globe_rows_match_term_by_term_globe7(tmp_path):
    exe = tmp_path / "nrl_rows_check"
    subprocess.run([NVCC, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", str(ROOT / "parahpop_b200" / "csrc"),
                    str(ROOT / "tests" / "nrl_rows_check.cu"), "-o", str(exe)], check=True)
    out = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    assert out["invalid_blocks"] == 0
    assert out["max_abs_diff"] < 1e-12, out
