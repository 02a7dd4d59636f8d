"""Build the in-tree native products of parahpop_b200 for sm_100a:

  parahpop_b200/lib/libparahpop_engine.so   C ABI (include/parahpop.h)
  parahpop_b200/bin/parahpop_gpu            reference-compatible command line

    python -m parahpop_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libparahpop_engine.so"
CLI = PKG / "bin" / "parahpop_gpu"
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["propagate.cu", "engine.cu", "peak.cu", "noalloc.cu", "server.cu", "nrl_diag.cu"]
# the step-kernel families: (object name, macro definitions)
INST = [("f64_grid", ["-DPHOP_T=double", "-DPHOP_SG=1"]), ("f64_mixed", ["-DPHOP_T=double", "-DPHOP_SG=0"]),
        ("f32_grid", ["-DPHOP_T=float", "-DPHOP_SG=1"]), ("f32_mixed", ["-DPHOP_T=float", "-DPHOP_SG=0"])]
CPP_SOURCES = ["value.cpp", "capi.cpp"]
HEADERS = ["propagate.cuh", "propagate_impl.cuh", "device_env.cuh", "nrlmsise00.cuh", "nrl_fast.cuh", "tide_field.cuh", "engine.hpp", "server.hpp", "value.hpp",
           "tables/nrlmsise00_coeffs.inc", "tables/tide_tables.inc"]


def _digest(cmd, deps) -> str:
    """Hash of a build step's command line and the contents of its inputs."""
    h = hashlib.sha256("\0".join(map(str, cmd)).encode())
    for d in deps:
        h.update(Path(d).read_bytes())
    return h.hexdigest()


def _stale(out: Path, cmd, deps) -> bool:
    """An output is rebuilt unless its stamp records the digest of exactly the
    inputs it was built from (content hashes, not modification times: an
    object compiled while a header was being edited is never taken as
    current)."""
    stamp = out.with_name(out.name + ".sha")
    return not out.exists() or not stamp.exists() or stamp.read_text() != _digest(cmd, deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout)
    return r.stdout


def _run_stamped(step):
    """Runs one compile step; the digest is taken before the compiler starts,
    so an input edited during the compile leaves the output stale."""
    cmd, out, deps = step
    digest = _digest(cmd, deps)
    stamp = out.with_name(out.name + ".sha")
    stamp.unlink(missing_ok=True)
    text = _run(cmd)
    stamp.write_text(digest)
    return text


def build(force: bool = False, jobs: int = 4, verbose_ptxas: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    CLI.parent.mkdir(exist_ok=True)
    hdrs = [SRC / h for h in HEADERS] + [PKG.parent / "include" / "parahpop.h"]
    steps = []
    objs = []
    for s in CU_SOURCES:
        o = OBJ / (s + ".o")
        objs.append(o)
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               "-I", str(SRC), "-c", str(SRC / s), "-o", str(o)]
        if force or _stale(o, cmd, [SRC / s] + hdrs):
            steps.append((cmd, o, [SRC / s] + hdrs))
    for sfx, defs in INST:
        o = OBJ / f"propagate_{sfx}.o"
        objs.append(o)
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               *defs, f"-DPHOP_SUFFIX={sfx}", "-I", str(SRC), "-c", str(SRC / "propagate_inst.cu"), "-o", str(o)]
        deps = [SRC / "propagate_inst.cu"] + hdrs
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        if force or _stale(o, cmd, deps):
            steps.append((cmd, o, deps))
    for s in CPP_SOURCES:
        o = OBJ / (s + ".o")
        objs.append(o)
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I", str(SRC), "-I", str(CUDA_HOME / "include"),
               "-c", str(SRC / s), "-o", str(o)]
        if force or _stale(o, cmd, [SRC / s] + hdrs):
            steps.append((cmd, o, [SRC / s] + hdrs))
    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        outs = list(ex.map(_run_stamped, steps))
    if verbose_ptxas:
        for o in outs:
            if "registers" in o:
                print(o)
    link = [NVCC, *ARCH, "-shared", *map(str, objs), "-o", str(LIB), "-Xlinker", "-soname=libparahpop_engine.so"]
    if force or steps or _stale(LIB, link, objs):
        _run_stamped((link, LIB, objs))
    main = SRC / "main_gpu.cpp"
    cli = ["g++", "-O2", str(main), "-o", str(CLI), "-L", str(LIB.parent), "-lparahpop_engine",
           "-Wl,-rpath,$ORIGIN/../lib"]
    if force or _stale(CLI, cli, [main, LIB]):
        _run_stamped((cli, CLI, [main, LIB]))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.ptxas))
