"""Python mirror of the reference's solver API over the C ABI.

``MPMSolver3D`` follows chains::MPMSolver3D (include/mpm_solver3d.h:21-96) and
``APICMPMSolver3D`` follows chains::APICMPMSolver3D
(include/apic_mpm_solver3d.h:20-92): same constructor arguments in the same
order (numpy arrays in place of thrust::host_vector<MaterialPoint3D>, tuples
in place of Eigen vectors), same method names, same sub-step split.  The
rendering methods (GL buffers, OpenVDB) are replaced by ``download``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check

InterpolationType = type("InterpolationType", (), {"LINEAR": 0, "QUADRATIC_BSPLINE": 1, "CUBIC_BSPLINE": 2})
ConstitutiveModel = type("ConstitutiveModel", (), {"FIXED_COROTATED": 0, "NEO_HOOKEAN": 1})


@dataclass
class Material:
    """Per-group snow material (src/material_point3d.cu:10-30 constructor arguments)."""
    youngs_modulus: float = 1.4e5
    poisson_ratio: float = 0.2
    hardening: float = 10.0
    critical_compression: float = 2.5e-2
    critical_stretch: float = 7.5e-3
    model: int = ConstitutiveModel.FIXED_COROTATED

    def to_c(self) -> _abi.Material:
        return _abi.Material(self.youngs_modulus, self.poisson_ratio, self.hardening, self.critical_compression,
                             self.critical_stretch, int(self.model))


@dataclass
class Particles:
    """Host particle set: the data of thrust::host_vector<MaterialPoint3D>.

    positions/velocities are (n, 3) float32; mass is (n,); material is (n,)
    uint16 indices into ``materials``; volume is only used with prescribed
    initial volumes.
    """
    positions: np.ndarray
    velocities: np.ndarray
    mass: np.ndarray
    materials: Sequence[Material] = field(default_factory=lambda: [Material()])
    material: Optional[np.ndarray] = None
    volume: Optional[np.ndarray] = None

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float32).reshape(-1, 3)
        n = self.positions.shape[0]
        self.velocities = np.ascontiguousarray(np.broadcast_to(np.asarray(self.velocities, np.float32), (n, 3)))
        self.mass = np.ascontiguousarray(np.broadcast_to(np.asarray(self.mass, np.float32), (n,)))
        if self.material is not None:
            self.material = np.ascontiguousarray(self.material, dtype=np.uint16)
        if self.volume is not None:
            self.volume = np.ascontiguousarray(np.broadcast_to(np.asarray(self.volume, np.float32), (n,)))

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    def to_c(self):
        """Returns (ParticlesIn, keepalive) for the C ABI."""
        mats = (_abi.Material * len(self.materials))(*[m.to_c() for m in self.materials])
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        pin = _abi.ParticlesIn()
        pin.n = self.n
        pin.position = fp(self.positions)
        pin.velocity = fp(self.velocities)
        pin.mass = fp(self.mass)
        pin.material = self.material.ctypes.data_as(C.POINTER(C.c_uint16)) if self.material is not None else None
        pin.volume = fp(self.volume)
        pin.materials = C.cast(mats, C.POINTER(_abi.Material))
        pin.nmaterials = len(self.materials)
        return pin, (mats, self)

    @staticmethod
    def concat(groups: Sequence["Particles"]) -> "Particles":
        """Stack groups (each with one material) the way the builder stacks
        particle groups (src/mpm_solver3d_builder.cu:66-73)."""
        mats, mids = [], []
        for g in groups:
            base = len(mats)
            mats.extend(g.materials)
            mids.append((g.material if g.material is not None else np.zeros(g.n, np.uint16)) + base)
        vol = None
        if all(g.volume is not None for g in groups) and groups:
            vol = np.concatenate([g.volume for g in groups])
        return Particles(np.concatenate([g.positions for g in groups]),
                         np.concatenate([g.velocities for g in groups]),
                         np.concatenate([g.mass for g in groups]), mats,
                         np.concatenate(mids).astype(np.uint16) if len(mats) > 1 else None, vol)


def scene_desc(origin, resolution, stride, friction, blend, interpolation, dt, *, transfer,
               gravity=9.80665, boundary=_abi.BOUNDARY_REFERENCE, sticky_cells=3,
               volume_mode=_abi.VOLUME_GRID_ESTIMATE, particles_collision=False) -> _abi.SceneDesc:
    d = _abi.SceneDesc()
    d.origin[:] = [float(v) for v in origin]
    d.resolution[:] = [int(v) for v in resolution]
    d.stride = float(stride)
    d.friction = float(friction)
    d.blend = float(blend)
    d.dt = float(dt)
    d.gravity = float(gravity)
    d.transfer = int(transfer)
    d.interpolation = int(interpolation)
    d.boundary = int(boundary)
    d.sticky_cells = int(sticky_cells)
    d.volume_mode = int(volume_mode)
    d.particles_collision = 1 if particles_collision else 0
    return d


class _SolverBase:
    _transfer = _abi.TRANSFER_PIC_FLIP

    def __init__(self, particles: Particles, gridOrigin, gridResolution, gridStride,
                 gridBoundaryFrictionCoefficient, blendCoefficient, interpolationType, deltaTime, **options):
        self._lib = _abi.load()
        if _abi.device_count() < 1:
            raise RuntimeError("mpm_b200 needs a CUDA device; there is no CPU fallback")
        device = options.pop("device", None)
        if device is not None:
            check(self._lib.mpm_set_device(int(device)), "mpm_set_device")
        self._desc = scene_desc(gridOrigin, gridResolution, gridStride, gridBoundaryFrictionCoefficient,
                                blendCoefficient, interpolationType, deltaTime, transfer=self._transfer, **options)
        self._n = particles.n
        self._res = tuple(int(r) for r in gridResolution)
        self._delta_time = float(deltaTime)
        self._blend_coefficient = float(blendCoefficient)
        pin, keep = particles.to_c()
        h = C.c_void_p()
        check(self._lib.mpm_solver_create(C.byref(self._desc), C.byref(pin), C.byref(h)), "mpm_solver_create")
        del keep
        self._h = h

    # -- checkpoints -------------------------------------------------------
    def save(self, path: str):
        """Write the full state to `path` (mpm_solver_save); resume with
        ``from_checkpoint``: the resumed steps are bitwise the ones this solver
        would take."""
        check(self._lib.mpm_solver_save(self._h, os.fsencode(path)), "save")

    @classmethod
    def from_checkpoint(cls, path: str, device: Optional[int] = None):
        lib = _abi.load()
        if _abi.device_count() < 1:
            raise RuntimeError("mpm_b200 needs a CUDA device; there is no CPU fallback")
        if device is not None:
            check(lib.mpm_set_device(int(device)), "mpm_set_device")
        h = C.c_void_p()
        check(lib.mpm_solver_load(os.fsencode(path), C.byref(h)), "mpm_solver_load")
        self = cls.__new__(cls)
        self._lib = lib
        self._h = h
        desc = _abi.SceneDesc()
        check(lib.mpm_solver_get_desc(h, C.byref(desc)), "get_desc")
        self._desc = desc
        n = C.c_size_t()
        check(lib.mpm_solver_num_particles(h, C.byref(n)), "num_particles")
        self._n = int(n.value)
        self._res = tuple(int(r) for r in desc.resolution)
        self._delta_time = float(desc.dt)
        self._blend_coefficient = float(desc.blend)
        return self

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.mpm_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- simulation (include/mpm_solver3d.h:37-63) -------------------------
    def simulateOneStep(self):
        check(self._lib.mpm_solver_step(self._h, 1), "simulateOneStep")

    def step(self, nsteps: int = 1):
        check(self._lib.mpm_solver_step(self._h, int(nsteps)), "step")

    def synchronize(self):
        check(self._lib.mpm_solver_synchronize(self._h), "synchronize")

    def switchIfEnableParticlesCollision(self):
        self._enable_particles_collision = not self._enable_particles_collision

    @property
    def _enable_particles_collision(self) -> bool:
        v = C.c_int32()
        check(self._lib.mpm_solver_get_particles_collision(self._h, C.byref(v)), "get_particles_collision")
        return bool(v.value)

    @_enable_particles_collision.setter
    def _enable_particles_collision(self, value: bool):
        check(self._lib.mpm_solver_set_particles_collision(self._h, 1 if value else 0), "set_particles_collision")

    def initialize(self):
        check(self._lib.mpm_solver_initialize(self._h), "initialize")

    def resetGrid(self):
        check(self._lib.mpm_solver_reset_grid(self._h), "resetGrid")

    def particlesToGrid(self):
        check(self._lib.mpm_solver_particles_to_grid(self._h), "particlesToGrid")

    def computeExternalForces(self):
        check(self._lib.mpm_solver_compute_external_forces(self._h), "computeExternalForces")

    def computeGravityForces(self):
        check(self._lib.mpm_solver_compute_gravity_forces(self._h), "computeGravityForces")

    def updateGridVelocities(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_update_grid_velocities(self._h, float(deltaTimeInSeconds)), "updateGridVelocities")

    def gridCollision(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_grid_collision(self._h, float(deltaTimeInSeconds)), "gridCollision")

    def solveLinearSystem(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_solve_linear_system(self._h, float(deltaTimeInSeconds)), "solveLinearSystem")

    def particlesCollision(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_particles_collision(self._h, float(deltaTimeInSeconds)), "particlesCollision")

    def advectParticles(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_advect_particles(self._h, float(deltaTimeInSeconds)), "advectParticles")

    # -- data --------------------------------------------------------------
    @property
    def num_particles(self) -> int:
        return self._n

    def download(self, field: int) -> np.ndarray:
        comps = _abi.FIELD_COMPONENTS[field]
        out = np.empty((self._n, comps), np.float32)
        check(self._lib.mpm_solver_download(self._h, int(field), out.ctypes.data_as(C.POINTER(C.c_float))),
              "download")
        return out.reshape(self._n, 3, 3) if comps == 9 else (out[:, 0] if comps == 1 else out)

    def upload(self, field: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float32)
        check(self._lib.mpm_solver_upload(self._h, int(field), a.ctypes.data_as(C.POINTER(C.c_float))), "upload")

    def download_grid(self, field: int) -> np.ndarray:
        comps = _abi.GRID_COMPONENTS[field]
        nodes = self._res[0] * self._res[1] * self._res[2]
        out = np.empty((nodes, comps), np.float32)
        check(self._lib.mpm_solver_download_grid(self._h, int(field), out.ctypes.data_as(C.POINTER(C.c_float))),
              "download_grid")
        return out[:, 0] if comps == 1 else out

    def positions(self) -> np.ndarray:
        return self.download(_abi.FIELD_POSITION)

    def velocities(self) -> np.ndarray:
        return self.download(_abi.FIELD_VELOCITY)

    def timed_step(self, nsteps: int) -> float:
        """Run nsteps steps timed by CUDA events on the solver's stream; returns ms."""
        ms = C.c_float()
        check(self._lib.mpm_solver_timed_step(self._h, int(nsteps), C.byref(ms)), "timed_step")
        return float(ms.value)

    def kernel_spans(self) -> dict:
        """Device-measured time per step (ms) of the P2G, grid and G2P launches
        inside the ordinary graph-replayed steps since the last call, and the
        number of steps: {family: (ms, steps)}."""
        nf = len(_abi.SPAN_FAMILIES)
        ms = (C.c_float * nf)()
        cnt = (C.c_int32 * nf)()
        check(self._lib.mpm_solver_kernel_spans(self._h, ms, cnt, nf), "mpm_solver_kernel_spans")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_abi.SPAN_FAMILIES)}

    def stats(self) -> dict:
        st = _abi.StepStats()
        check(self._lib.mpm_solver_stats(self._h, C.byref(st)), "stats")
        return dict(active_blocks=st.active_blocks, outside_blocks=st.outside_blocks, active_nodes=st.active_nodes)

    # ---- launch settings (no counterpart in the reference) -----------------
    def tuning(self) -> dict:
        """Launch settings of the step kernels: particles per G2P work item,
        particles staged per P2G pass (0 = chosen from density) and the
        largest P2G work item taken by a single warp (0 = none, -1 = chosen
        from the item counts)."""
        t = _abi.Tuning()
        check(self._lib.mpm_solver_get_tuning(self._h, C.byref(t)), "get_tuning")
        return dict(g2p_chunk=t.g2p_chunk, p2g_stage=t.p2g_stage, p2g_warp_max=t.p2g_warp_max)

    def set_tuning(self, g2p_chunk: int = 1024, p2g_stage: int = 0, p2g_warp_max: int = -1):
        """Set the launch settings; results are bitwise the same for any."""
        t = _abi.Tuning(int(g2p_chunk), int(p2g_stage), int(p2g_warp_max))
        check(self._lib.mpm_solver_set_tuning(self._h, C.byref(t)), "set_tuning")

    def autotune(self, steps_per_candidate: int = 3, force: bool = False, use_disk: bool = True) -> dict:
        """Choose the launch settings for this scene's (stencil, transfer,
        particles-per-cell bucket) from the tuning cache, or by timing the
        candidates over real steps of the simulation (which advance it).
        Returns the chosen settings and the number of steps taken."""
        flags = (_abi.TUNE_FORCE if force else 0) | (0 if use_disk else _abi.TUNE_NO_DISK)
        run = C.c_int32(0)
        check(self._lib.mpm_solver_autotune(self._h, int(steps_per_candidate), flags, C.byref(run)), "autotune")
        return dict(self.tuning(), steps=int(run.value))

    def download_into(self, field: int, ptr: int):
        """Download into caller memory at address ptr (e.g. pinned host memory)."""
        check(self._lib.mpm_solver_download(self._h, int(field), C.cast(C.c_void_p(ptr), C.POINTER(C.c_float))),
              "download")

    def download_async(self, field: int, ptr: int):
        """Queue a download of the current state into caller memory at address
        ptr (pinned host memory to overlap later steps); the data is complete
        after download_wait() or synchronize()."""
        check(self._lib.mpm_solver_download_async(self._h, int(field), C.c_void_p(ptr)), "download_async")

    def density(self) -> np.ndarray:
        """Density grid sum_p m_p w_ip / h^3 of the current state (the grid the
        reference's writeToOpenVDB writes), shape (res_z, res_y, res_x)."""
        out = np.empty(self._res[0] * self._res[1] * self._res[2], np.float32)
        check(self._lib.mpm_solver_download_density(self._h, out.ctypes.data_as(C.POINTER(C.c_float))), "density")
        return out.reshape(self._res[2], self._res[1], self._res[0])

    def writeToOpenVDB(self, filePath: str):
        """OpenVDB file of the density grid of the current state: one FloatGrid
        "density" (MPMSolver3D::writeToOpenVDB, src/mpm_solver3d.cu:509-572)."""
        check(self._lib.mpm_solver_write_vdb(self._h, os.fsencode(filePath)), "writeToOpenVDB")

    write_vdb = writeToOpenVDB

    def download_wait(self):
        check(self._lib.mpm_solver_download_wait(self._h), "download_wait")

    def set_implicit(self, beta: float, max_iter: int = 50, tol: float = 1e-5):
        """Semi-implicit update: beta > 0 solves (M + beta dt^2 H) v = M v* every
        step (1/2 semi-implicit, 1 backward Euler); 0 is the explicit step."""
        check(self._lib.mpm_solver_set_implicit(self._h, float(beta), int(max_iter), float(tol)), "set_implicit")

    def solve_info(self) -> tuple:
        """(iterations, |r| / |M v*|) of the last semi-implicit solve."""
        it, res = C.c_int32(), C.c_float()
        check(self._lib.mpm_solver_solve_info(self._h, C.byref(it), C.byref(res)), "solve_info")
        return it.value, res.value

    def set_cfl(self, cfl: float):
        """CFL time step: cfl > 0 makes each step's dt min(dt, cfl h / max|v_p|); 0 restores the fixed dt."""
        check(self._lib.mpm_solver_set_cfl(self._h, float(cfl)), "set_cfl")

    def time(self) -> tuple:
        """(simulated time advanced by step(), dt of the last step)."""
        t, dt = C.c_double(), C.c_float()
        check(self._lib.mpm_solver_time(self._h, C.byref(t), C.byref(dt)), "time")
        return t.value, dt.value

    def set_collision_object(self, obj=None):
        """Level-set collision object (mpm_b200.level_set.LevelSetCollisionObject3D)
        applied in every grid collision; None removes it."""
        if obj is None:
            check(self._lib.mpm_solver_set_level_set(self._h, None, 0.0, None), "set_level_set")
            return
        phi, vel = obj.arrays(self._res)
        F = C.POINTER(C.c_float)
        check(self._lib.mpm_solver_set_level_set(self._h, phi.ctypes.data_as(F), float(obj.friction),
                                                 vel.ctypes.data_as(F)), "set_level_set")

    def profile(self, enable: bool = True):
        check(self._lib.mpm_solver_profile(self._h, 1 if enable else 0), "profile")

    def profile_read(self) -> dict:
        nf = len(_abi.KERNEL_FAMILIES)
        ms = (C.c_float * nf)()
        cnt = (C.c_int32 * nf)()
        check(self._lib.mpm_solver_profile_read(self._h, ms, cnt, nf), "profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_abi.KERNEL_FAMILIES)}

    # snake_case aliases
    simulate_one_step = simulateOneStep
    reset_grid = resetGrid
    particles_to_grid = particlesToGrid
    compute_external_forces = computeExternalForces
    update_grid_velocities = updateGridVelocities
    grid_collision = gridCollision
    particles_collision = particlesCollision
    advect_particles = advectParticles


class MPMSolver3D(_SolverBase):
    """PIC-FLIP solver (include/mpm_solver3d.h:25-34 argument order)."""
    _transfer = _abi.TRANSFER_PIC_FLIP

    def gridToParticles(self, deltaTimeInSeconds: float, blendCoefficient: float):
        check(self._lib.mpm_solver_grid_to_particles(self._h, float(deltaTimeInSeconds), float(blendCoefficient)),
              "gridToParticles")

    grid_to_particles = gridToParticles


class APICMPMSolver3D(_SolverBase):
    """APIC solver (include/apic_mpm_solver3d.h:24-32 argument order: no blend)."""
    _transfer = _abi.TRANSFER_APIC

    def __init__(self, particles: Particles, gridOrigin, gridResolution, gridStride,
                 gridBoundaryFrictionCoefficient, interpolationType, deltaTime, **options):
        super().__init__(particles, gridOrigin, gridResolution, gridStride, gridBoundaryFrictionCoefficient, 0.0,
                         interpolationType, deltaTime, **options)

    def gridToParticles(self, deltaTimeInSeconds: float):
        check(self._lib.mpm_solver_grid_to_particles(self._h, float(deltaTimeInSeconds), 0.0), "gridToParticles")

    grid_to_particles = gridToParticles
