"""Builds libcgef_b200.so in place: the CUDA kernels and the C ABI, for sm_100a.

    python -m cgef_b200.build          (from coarsegrainingenergyfluxes.jl_b200/)

nvcc cross-compiles without a GPU; the library lands next to this file, where ``_lib`` loads it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO_ROOT, "include")
LIB_PATH = os.path.join(HERE, "libcgef_b200.so")
PEAK_LIB_PATH = os.path.join(HERE, "libcgef_peak.so")
SOURCES = ["kernels.cu", "rowspec.cu", "cgef_api.cu", "noalloc.cu", "closure.cu", "decomposition.cu", "pipeline.cu",
           "plan_build.cpp"]
HEADERS = ["cgef_internal.h", "banded_common.cuh"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "cgef_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build_peak_probe(force: bool = False) -> str:
    """libcgef_peak.so: the FP64 FMA throughput probe the benchmark uses as its roofline peak."""
    src = os.path.join(CSRC, "peak_probe.cu")
    if not force and os.path.exists(PEAK_LIB_PATH) and os.path.getmtime(PEAK_LIB_PATH) >= os.path.getmtime(src):
        return PEAK_LIB_PATH
    cmd = [_nvcc(), "-ccbin", os.environ.get("NVCC_CCBIN", "/usr/bin/g++"), "-O3",
           "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared", src,
           "-o", PEAK_LIB_PATH + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcgef_peak.so")
    os.replace(PEAK_LIB_PATH + ".tmp", PEAK_LIB_PATH)
    return PEAK_LIB_PATH


def build(verbose: bool = False, force: bool = False, out: str = LIB_PATH, defines=()) -> str:
    """Compiles the library to `out` (default: in place); `defines` are extra -D tuning macros."""
    if not force and out == LIB_PATH and not needs_build():
        return out
    cmd = [
        _nvcc(), "-O3", "-std=c++17",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo", "--fmad=false",
        "-Xcompiler", "-fPIC", "-shared",
        "-I", INCLUDE, "-I", CSRC,
        *[f"-D{d}" for d in defines],
        *[os.path.join(CSRC, s) for s in SOURCES],
        "-o", out + ".tmp",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    env = dict(os.environ)
    env.setdefault("NVCC_CCBIN", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
    cmd[1:1] = ["-ccbin", env["NVCC_CCBIN"]]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcgef_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
    print(build_peak_probe(force=True))
