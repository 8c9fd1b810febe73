"""Reference-naive GPU baseline: build and ctypes binding.

``naive_mpm.cu`` keeps the reference's execution model (AoS particles and
52 B grid nodes, one thread per particle or node, seven float atomicAdd per
(particle, node) in P2G, per-node double-literal spline evaluation, two SVDs
per particle, one synchronised launch per sub-step).  It is a measuring stick
for the B200 engine, not part of the library: only ``bench.py`` and the tests
load it.

    python baseline/naive/naive.py      # build libmpm_naive.so in place
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "naive_mpm.cu")
LIB = os.path.join(HERE, "libmpm_naive.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
DEPS = [SRC, os.path.join(ROOT, "include", "mpm_b200.h"), os.path.join(ROOT, "mpm_b200", "csrc", "mpm_math.cuh")]


def build(verbose: bool = False) -> str:
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in DEPS):
        return LIB
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", SRC, "-o", LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("naive baseline build failed:\n" + r.stdout)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is not built (python baseline/naive/naive.py)")
        lib = C.CDLL(LIB)
        lib.naive_last_error.restype = C.c_char_p
        lib.naive_create.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
        lib.naive_destroy.argtypes = [C.c_void_p]
        lib.naive_step.argtypes = [C.c_void_p, C.c_int32]
        lib.naive_timed_step.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]
        lib.naive_download.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        _lib = lib
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: status {rc}: {load().naive_last_error().decode()}")


class NaiveSolver:
    """One scene on the naive baseline; same descriptor and particles as the
    library's solvers (``mpm_b200.scenes.Scene.desc()`` / ``.particles``)."""

    def __init__(self, desc, particles):
        lib = load()
        self.n = len(particles.mass)
        pin, self._keep = particles.to_c()
        self._desc = desc
        self.h = C.c_void_p()
        _check(lib.naive_create(C.byref(desc), C.byref(pin), C.byref(self.h)), "naive_create")

    def step(self, n=1):
        _check(load().naive_step(self.h, n), "naive_step")

    def timed_step(self, n):
        ms = C.c_float()
        _check(load().naive_timed_step(self.h, n, C.byref(ms)), "naive_timed_step")
        return ms.value

    def download(self, field):
        from mpm_b200 import _abi
        comps = {_abi.FIELD_POSITION: 3, _abi.FIELD_VELOCITY: 3, _abi.FIELD_FE: 9, _abi.FIELD_FP: 9,
                 _abi.FIELD_B: 9, _abi.FIELD_VOLUME0: 1, _abi.FIELD_MASS: 1}[field]
        out = np.empty((self.n, comps), dtype=np.float32)
        _check(load().naive_download(self.h, field, out.ctypes.data), "naive_download")
        return out if comps > 1 else out[:, 0]

    def close(self):
        if self.h:
            load().naive_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


if __name__ == "__main__":
    print(build(verbose=True))
