"""Builds libcgef_b200.so in place: the CUDA kernels and the C ABI, for sm_100a.

    python -m cgef_b200.build          (from coarsegrainingenergyfluxes.jl_b200/)

nvcc cross-compiles without a GPU; the library lands next to this file, where ``_lib`` loads it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO_ROOT, "include")
LIB_PATH = os.path.join(HERE, "libcgef_b200.so")
PEAK_LIB_PATH = os.path.join(HERE, "libcgef_peak.so")
SOURCES = ["kernels.cu", "rowspec.cu", "cgef_api.cu", "noalloc.cu", "closure.cu", "decomposition.cu", "pipeline.cu",
           "plan_build.cpp", "plan_device.cu", "pi_w.cu"]
HEADERS = ["cgef_internal.h", "banded_common.cuh", "stencil.cuh"]


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
    """Compiles the library to `out` (default: in place); `defines` are extra -D tuning macros.  The
    sources compile in parallel to objects in a temporary directory, then link into one shared library."""
    if not force and out == LIB_PATH and not needs_build():
        return out
    env = dict(os.environ)
    env.setdefault("NVCC_CCBIN", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
    common = [
        _nvcc(), "-ccbin", env["NVCC_CCBIN"], "-O3", "-std=c++17",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo", "--fmad=false",
        "-Xcompiler", "-fPIC",
        "-I", INCLUDE, "-I", CSRC,
        *[f"-D{d}" for d in defines],
    ]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    with tempfile.TemporaryDirectory(prefix="cgef_build_") as tmp:
        objs = [os.path.join(tmp, os.path.splitext(s)[0] + ".o") for s in SOURCES]

        def compile_one(k: int):
            return subprocess.run(common + ["-c", os.path.join(CSRC, SOURCES[k]), "-o", objs[k]],
                                  capture_output=True, text=True, env=env)

        with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
            results = list(ex.map(compile_one, range(len(SOURCES))))
        for r in results:
            if r.returncode != 0 or verbose:
                sys.stderr.write(r.stdout + r.stderr)
        if any(r.returncode != 0 for r in results):
            raise RuntimeError("nvcc failed building libcgef_b200.so")
        link = [_nvcc(), "-ccbin", env["NVCC_CCBIN"], "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                *objs, "-o", out + ".tmp"]
        r = subprocess.run(link, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed linking libcgef_b200.so")
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
    print(build_peak_probe(force=True))
