"""Build the in-tree shared library ``libhfm_b200.so`` (C ABI of include/hfm_b200.h) and the
FileHFM-compatible command-line front-end, for sm_100a only.

    python -m hamiltonfastmarching_b200.build [--force] [--jobs N]

Each CUDA translation unit is compiled separately (parallel) with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false`` and linked with the static CUDA runtime,
so the library carries no dependency on torch. Outputs live next to this file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "hfm_b200")
LIB = os.path.join(HERE, "libhfm_b200.so")
CLI = os.path.join(HERE, "bin", "FileHFM_b200")

SOURCES = ["io.cpp", "run.cu", "eulerian.cu", "curvature.cu", "runtime.cu", "static_scratch.cu", "server.cu"]
CLI_SOURCES = ["cli/FileHFM.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags(extra=()):
    # -fmad=false: device arithmetic rounds every product and sum, as the reference's x86-64 build
    # does (no fused multiply-add); the Selling decompositions of the TTI3 path depend on it
    return ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
            "-I", os.path.join(ROOT, "include"), *ARCH, *extra]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "hfm_b200.h"))
    return hs


def _compile(src, force):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    if not force and not _stale(obj, [path] + _headers()):
        return obj
    cmd = [nvcc(), "-c", "-x", "cu", path, "-o", obj, *_flags()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 4, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", *ARCH, "-o", LIB + ".tmp", *objs, "-cudart", "static", "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    cli_src = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    if all(os.path.exists(s) for s in cli_src) and (force or _stale(CLI, cli_src + [LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), *cli_src, "-o", CLI,
               "-L", HERE, "-lhfm_b200", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=4)
    a = ap.parse_args(argv)
    build(force=a.force, jobs=a.jobs, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
