"""Build the sm_100a shared library ``mpm_b200/libmpm_b200.so`` in-tree.

Every CUDA source under ``mpm_b200/csrc`` is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into
one shared library whose exported symbols are the C ABI of
``include/mpm_b200.h`` and ``include/mpm_b200_batch.h``.  Objects are rebuilt
only when a source or header is newer than them.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmpm_b200.so")
CLI = os.path.join(HERE, "mpm-run")
# Host compiler of the CLI: the system g++ (a CXX from the environment may be a
# wrapper without the full C++ runtime); override with MPM_HOSTCXX.
HOSTCXX = os.environ.get("MPM_HOSTCXX", "/usr/bin/g++")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-Xcompiler", "-ffp-contract=off"]

# Extra nvcc flags (space separated) for builds of variants, e.g. a -D of a
# launch-bound setting.
EXTRA = os.environ.get("MPM_NVCC_EXTRA", "").split()

SOURCES = ["sort.cu", "kernels.cu", "implicit.cu", "engine.cu", "sort_noalloc.cu", "config.cpp", "vdb.cpp"]


def _headers():
    hs = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                hs.append(os.path.join(d, f))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            jobs.append([NVCC, *ARCH, *FLAGS, *EXTRA, "-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], verbose)
    # headless driver over the C++ facade (include/chains/mpm_b200.hpp)
    src = os.path.join(CSRC, "mpm_run.cpp")
    if _stale(CLI, [src, LIB] + headers):
        _run([HOSTCXX, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", CLI, "-L", HERE,
              "-lmpm_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
