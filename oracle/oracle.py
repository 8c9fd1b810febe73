"""ctypes wrapper of the CPU oracle (oracle/mpm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the mpm_b200 package.  Parity unpinned against
an executed reference (the reference does not build here); see mpm_oracle.hpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    from mpm_b200 import _abi
    lib = C.CDLL(LIB)
    P, D = C.c_void_p, C.POINTER(C.c_double)
    sig = {
        "orc_solver_create": (P, [C.c_int, C.POINTER(_abi.SceneDesc), C.POINTER(_abi.ParticlesIn)]),
        "orc_solver_destroy": (None, [P]),
        "orc_set_threads": (None, [P, C.c_int]),
        "orc_set_particles_collision": (None, [P, C.c_int]),
        "orc_initialize": (None, [P]),
        "orc_reset_grid": (None, [P]),
        "orc_particles_to_grid": (None, [P]),
        "orc_gravity": (None, [P]),
        "orc_update_grid_velocities": (None, [P, C.c_double]),
        "orc_grid_collision": (None, [P, C.c_double]),
        "orc_grid_to_particles": (None, [P, C.c_double, C.c_double]),
        "orc_particles_collision": (None, [P, C.c_double]),
        "orc_advect": (None, [P, C.c_double]),
        "orc_step": (None, [P, C.c_int]),
        "orc_get_particles": (C.c_int, [P, C.c_int, D]),
        "orc_set_particles": (C.c_int, [P, C.c_int, D]),
        "orc_get_grid": (C.c_int, [P, C.c_int, D]),
        "orc_spline": (None, [C.c_int, C.c_int, D, C.c_int, D, D]),
        "orc_svd3": (None, [C.c_int, D, D, D, D]),
        "orc_collision": (None, [C.c_int, D, D, D, D, C.c_double, D]),
        "orc_set_level_set": (C.c_int, [P, D, C.c_double, D]),
        "orc_set_cfl": (None, [P, C.c_double]),
        "orc_set_implicit": (None, [P, C.c_double, C.c_int, C.c_double]),
        "orc_solve_linear_system": (None, [P, C.c_double]),
        "orc_solve_info": (None, [P, C.POINTER(C.c_int), D]),
        "orc_grid_operator": (None, [P, C.c_int, D, D]),
        "orc_time": (None, [P, D, D]),
        "orc_level_set_collision": (None, [C.c_int, C.POINTER(C.c_int), D, C.c_double, D, C.c_double, D, D, D, D]),
        "orc_stress": (None, [C.c_int, C.c_int, D, D, C.c_double, C.c_double, C.c_double, C.c_double, D, D]),
        "orc_update_deformation": (None, [C.c_int, D, D, D, C.c_double, C.c_double, C.c_double]),
        "orc_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


PARTICLE_COMPONENTS = {0: 3, 1: 3, 2: 9, 3: 9, 4: 9, 5: 1, 6: 1, 8: 1, 9: 1}
GRID_COMPONENTS = {0: 1, 1: 3, 2: 3, 3: 3}


class OracleSolver:
    """CPU restatement of MPMSolver3D / APICMPMSolver3D (bits = 32: reference
    restatement in float; bits = 64: FP64 oracle)."""

    def __init__(self, desc, particles, bits: int = 64, threads: int = 1):
        self.lib = load()
        pin, keep = particles.to_c()
        self.h = self.lib.orc_solver_create(bits, C.byref(desc), C.byref(pin))
        if not self.h:
            raise RuntimeError("oracle create failed: " + self.lib.orc_last_error().decode())
        del keep
        self.n = particles.n
        self.res = tuple(desc.resolution)
        self.desc = desc
        self.lib.orc_set_threads(self.h, int(threads))
        self.lib.orc_set_particles_collision(self.h, int(desc.particles_collision))
        self.lib.orc_initialize(self.h)

    def close(self):
        if self.h:
            self.lib.orc_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, t):
        self.lib.orc_set_threads(self.h, int(t))

    def set_particles_collision(self, on: bool):
        self.lib.orc_set_particles_collision(self.h, 1 if on else 0)

    def set_level_set(self, phi=None, friction: float = 0.0, velocity=(0.0, 0.0, 0.0)):
        """Level-set collision object (signed distance per grid node), None removes it."""
        if phi is None:
            self.lib.orc_set_level_set(self.h, None, 0.0, None)
            return
        phi = np.ascontiguousarray(phi, np.float64).reshape(-1)
        assert phi.size == self.res[0] * self.res[1] * self.res[2]
        vel = np.ascontiguousarray(velocity, np.float64).reshape(3)
        if self.lib.orc_set_level_set(self.h, _dp(phi), float(friction), _dp(vel)):
            raise ValueError(self.lib.orc_last_error().decode())

    def set_implicit(self, beta: float, max_iter: int = 30, tol: float = 1e-5):
        self.lib.orc_set_implicit(self.h, float(beta), int(max_iter), float(tol))

    def solve_linear_system(self, dt):
        self.lib.orc_solve_linear_system(self.h, float(dt))

    def solve_info(self) -> tuple:
        it, res = C.c_int(), np.zeros(1)
        self.lib.orc_solve_info(self.h, C.byref(it), _dp(res))
        return it.value, float(res[0])

    def hessian_action(self, u) -> np.ndarray:
        return self._grid_op(0, u)

    def displaced_force(self, d) -> np.ndarray:
        return self._grid_op(1, d)

    def _grid_op(self, which, u):
        u = np.ascontiguousarray(u, np.float64).reshape(-1, 3)
        assert u.shape[0] == self.res[0] * self.res[1] * self.res[2]
        out = np.empty_like(u)
        self.lib.orc_grid_operator(self.h, int(which), _dp(u), _dp(out))
        return out

    def set_cfl(self, cfl: float):
        self.lib.orc_set_cfl(self.h, float(cfl))

    def time(self) -> tuple:
        t, dt = np.zeros(1), np.zeros(1)
        self.lib.orc_time(self.h, _dp(t), _dp(dt))
        return float(t[0]), float(dt[0])

    def step(self, n=1):
        self.lib.orc_step(self.h, int(n))

    def initialize(self):
        self.lib.orc_initialize(self.h)

    def reset_grid(self):
        self.lib.orc_reset_grid(self.h)

    def particles_to_grid(self):
        self.lib.orc_particles_to_grid(self.h)

    def gravity(self):
        self.lib.orc_gravity(self.h)

    def update_grid_velocities(self, dt):
        self.lib.orc_update_grid_velocities(self.h, dt)

    def grid_collision(self, dt):
        self.lib.orc_grid_collision(self.h, dt)

    def grid_to_particles(self, dt, blend):
        self.lib.orc_grid_to_particles(self.h, dt, blend)

    def particles_collision(self, dt):
        self.lib.orc_particles_collision(self.h, dt)

    def advect(self, dt):
        self.lib.orc_advect(self.h, dt)

    def get(self, field: int) -> np.ndarray:
        c = PARTICLE_COMPONENTS[field]
        out = np.empty((self.n, c), np.float64)
        if self.lib.orc_get_particles(self.h, field, _dp(out)):
            raise ValueError(field)
        return out.reshape(self.n, 3, 3) if c == 9 else (out[:, 0] if c == 1 else out)

    def set(self, field: int, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        if self.lib.orc_set_particles(self.h, field, _dp(a)):
            raise ValueError(field)

    def grid(self, field: int) -> np.ndarray:
        c = GRID_COMPONENTS[field]
        nodes = self.res[0] * self.res[1] * self.res[2]
        out = np.empty((nodes, c), np.float64)
        if self.lib.orc_get_grid(self.h, field, _dp(out)):
            raise ValueError(field)
        return out[:, 0] if c == 1 else out


def spline(bits: int, kind: int, x) -> tuple:
    lib = load()
    x = np.ascontiguousarray(x, np.float64)
    N = np.empty_like(x)
    dN = np.empty_like(x)
    lib.orc_spline(bits, kind, _dp(x), x.size, _dp(N), _dp(dN))
    return N, dN


def svd3(A, mode: int = 2):
    """mode 0: McAdams float, 1: McAdams double, 2: exact double."""
    lib = load()
    A = np.ascontiguousarray(A, np.float64).reshape(9)
    U, s, V = np.empty(9), np.empty(3), np.empty(9)
    lib.orc_svd3(mode, _dp(A), _dp(U), _dp(s), _dp(V))
    return U.reshape(3, 3), s, V.reshape(3, 3)


def collision(bits, pos, vel, lo, hi, friction):
    lib = load()
    a = [np.ascontiguousarray(v, np.float64) for v in (pos, vel, lo, hi)]
    out = np.empty(3)
    lib.orc_collision(bits, *[_dp(v) for v in a], float(friction), _dp(out))
    return out


def level_set_collision(bits, res, origin, h, phi, friction, vco, pos, vel):
    lib = load()
    r = (C.c_int * 3)(*[int(v) for v in res])
    a = [np.ascontiguousarray(v, np.float64).reshape(-1) for v in (origin, phi, vco, pos, vel)]
    out = np.empty(3)
    lib.orc_level_set_collision(bits, r, _dp(a[0]), float(h), _dp(a[1]), float(friction), _dp(a[2]), _dp(a[3]),
                                _dp(a[4]), _dp(out))
    return out


def stress(bits, model, Fe, Fp, mu0, la0, xi, V0):
    lib = load()
    Fe = np.ascontiguousarray(Fe, np.float64).reshape(9)
    Fp = np.ascontiguousarray(Fp, np.float64).reshape(9)
    out, Fe_out = np.empty(9), np.empty(9)
    lib.orc_stress(bits, model, _dp(Fe), _dp(Fp), mu0, la0, xi, V0, _dp(out), _dp(Fe_out))
    return out.reshape(3, 3), Fe_out.reshape(3, 3)


def update_deformation(bits, Fe, Fp, gradv, dt, theta_c, theta_s):
    lib = load()
    Fe = np.ascontiguousarray(Fe, np.float64).reshape(9).copy()
    Fp = np.ascontiguousarray(Fp, np.float64).reshape(9).copy()
    g = np.ascontiguousarray(gradv, np.float64).reshape(9)
    lib.orc_update_deformation(bits, _dp(Fe), _dp(Fp), _dp(g), dt, theta_c, theta_s)
    return Fe.reshape(3, 3), Fp.reshape(3, 3)
