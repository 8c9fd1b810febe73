"""Batched scenes over the C ABI of include/mpm_b200_batch.h.

A Batch advances many independent scenes -- different particle counts,
grids, transfers, splines and materials -- with one launch sequence per step
(sort, block compaction, P2G, grid pass, G2P over the active blocks of every
scene).  Scenes can be added and removed between steps; the serving loop
(mpm_b200.serving) uses that for continuous batching.  The reference has no
batching; each scene's result is bitwise the result of solving it alone.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict

import numpy as np

from . import _abi
from ._abi import check


class Batch:
    def __init__(self, device: int | None = None):
        self._lib = _abi.load()
        if _abi.device_count() < 1:
            raise RuntimeError("mpm_b200 needs a CUDA device; there is no CPU fallback")
        if device is not None:
            check(self._lib.mpm_set_device(int(device)), "mpm_set_device")
        h = C.c_void_p()
        check(self._lib.mpm_batch_create(C.byref(h)), "mpm_batch_create")
        self._h = h
        self._n: Dict[int, int] = {}
        self._res: Dict[int, tuple] = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mpm_batch_destroy(self._h)
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

    def add(self, scene) -> int:
        """Add a mpm_b200.scenes.Scene; returns its id."""
        desc = scene.desc()
        pin, keep = scene.particles.to_c()
        sid = C.c_int32()
        check(self._lib.mpm_batch_add_scene(self._h, C.byref(desc), C.byref(pin), C.byref(sid)),
              "mpm_batch_add_scene")
        del keep
        self._n[int(sid.value)] = scene.n
        self._res[int(sid.value)] = tuple(int(r) for r in scene.resolution)
        return int(sid.value)

    def remove(self, sid: int):
        check(self._lib.mpm_batch_remove_scene(self._h, int(sid)), "mpm_batch_remove_scene")
        self._n.pop(int(sid), None)

    def save_scene(self, sid: int, path: str):
        """Checkpoint one scene (the format of MPMSolver3D.save)."""
        check(self._lib.mpm_batch_save_scene(self._h, int(sid), os.fsencode(path)), "mpm_batch_save_scene")

    def load_scene(self, path: str) -> int:
        """Add a scene from a checkpoint; returns its id."""
        sid = C.c_int32()
        check(self._lib.mpm_batch_load_scene(self._h, os.fsencode(path), C.byref(sid)), "mpm_batch_load_scene")
        n = C.c_size_t()
        check(self._lib.mpm_batch_scene_particles(self._h, sid, C.byref(n)), "mpm_batch_scene_particles")
        desc = _abi.SceneDesc()
        check(self._lib.mpm_batch_scene_desc(self._h, sid, C.byref(desc)), "mpm_batch_scene_desc")
        self._n[int(sid.value)] = int(n.value)
        self._res[int(sid.value)] = tuple(int(r) for r in desc.resolution)
        return int(sid.value)

    @property
    def num_scenes(self) -> int:
        return len(self._n)

    @property
    def num_particles(self) -> int:
        return int(sum(self._n.values()))

    def step(self, nsteps: int = 1):
        check(self._lib.mpm_batch_step(self._h, int(nsteps)), "mpm_batch_step")

    def synchronize(self):
        check(self._lib.mpm_batch_synchronize(self._h), "mpm_batch_synchronize")

    def timed_step(self, nsteps: int) -> float:
        ms = C.c_float()
        check(self._lib.mpm_batch_timed_step(self._h, int(nsteps), C.byref(ms)), "mpm_batch_timed_step")
        return float(ms.value)

    def download(self, sid: int, field: int) -> np.ndarray:
        n = self._n[int(sid)]
        comps = _abi.FIELD_COMPONENTS[field]
        out = np.empty((n, comps), np.float32)
        check(self._lib.mpm_batch_download(self._h, int(sid), int(field), out.ctypes.data_as(C.POINTER(C.c_float))),
              "mpm_batch_download")
        return out.reshape(n, 3, 3) if comps == 9 else (out[:, 0] if comps == 1 else out)

    def density(self, sid: int) -> np.ndarray:
        """Density grid of one scene (see MPMSolver3D.density), shape (res_z, res_y, res_x)."""
        res = self._res[int(sid)]
        out = np.empty(res[0] * res[1] * res[2], np.float32)
        check(self._lib.mpm_batch_download_density(self._h, int(sid), out.ctypes.data_as(C.POINTER(C.c_float))),
              "mpm_batch_download_density")
        return out.reshape(res[2], res[1], res[0])

    def time_steps(self, enable: bool = True):
        """Bracket every step with events so that step_times() can report device
        step times without synchronizing (for serving loops)."""
        check(self._lib.mpm_batch_time_steps(self._h, 1 if enable else 0), "mpm_batch_time_steps")

    def step_times(self, capacity: int = 256) -> list:
        """Device times (ms) of the timed steps completed since the last call,
        oldest first; does not wait."""
        out, got = [], capacity
        buf = (C.c_float * capacity)()
        while got == capacity:
            n = C.c_int32(0)
            check(self._lib.mpm_batch_step_times(self._h, buf, capacity, C.byref(n)), "mpm_batch_step_times")
            got = int(n.value)
            out.extend(buf[:got])
        return out

    def wait_steps(self, in_flight: int = 1):
        """Block until at most `in_flight` timed steps are queued or running."""
        check(self._lib.mpm_batch_wait_steps(self._h, int(in_flight)), "mpm_batch_wait_steps")

    def write_vdb(self, sid: int, path: str):
        """OpenVDB file of one scene's density grid (see MPMSolver3D.writeToOpenVDB)."""
        check(self._lib.mpm_batch_write_vdb(self._h, int(sid), os.fsencode(path)), "mpm_batch_write_vdb")

    def set_implicit(self, sid: int, beta: float, max_iter: int = 50, tol: float = 1e-5):
        """Semi-implicit update of one scene (see MPMSolver3D.set_implicit)."""
        check(self._lib.mpm_batch_set_implicit(self._h, int(sid), float(beta), int(max_iter), float(tol)),
              "mpm_batch_set_implicit")

    def solve_info(self, sid: int) -> tuple:
        it, res = C.c_int32(), C.c_float()
        check(self._lib.mpm_batch_solve_info(self._h, int(sid), C.byref(it), C.byref(res)), "mpm_batch_solve_info")
        return it.value, res.value

    def set_cfl(self, sid: int, cfl: float):
        """CFL time step of one scene (see MPMSolver3D.set_cfl)."""
        check(self._lib.mpm_batch_set_cfl(self._h, int(sid), float(cfl)), "mpm_batch_set_cfl")

    def time(self, sid: int) -> tuple:
        """(simulated time, dt of the last step) of one scene."""
        t, dt = C.c_double(), C.c_float()
        check(self._lib.mpm_batch_time(self._h, int(sid), C.byref(t), C.byref(dt)), "mpm_batch_time")
        return t.value, dt.value

    def set_collision_object(self, sid: int, obj=None):
        """Level-set collision object of one scene (see MPMSolver3D.set_collision_object)."""
        F = C.POINTER(C.c_float)
        if obj is None:
            check(self._lib.mpm_batch_set_level_set(self._h, int(sid), None, 0.0, None), "mpm_batch_set_level_set")
            return
        phi, vel = obj.arrays(self._res[int(sid)])
        check(self._lib.mpm_batch_set_level_set(self._h, int(sid), phi.ctypes.data_as(F), float(obj.friction),
                                                vel.ctypes.data_as(F)), "mpm_batch_set_level_set")

    def download_async(self, sid: int, field: int, ptr: int):
        """Queue a download of one scene's current state into caller memory at
        address ptr; complete after download_wait() or synchronize()."""
        check(self._lib.mpm_batch_download_async(self._h, int(sid), int(field), C.c_void_p(ptr)),
              "mpm_batch_download_async")

    def download_wait(self):
        check(self._lib.mpm_batch_download_wait(self._h), "mpm_batch_download_wait")

    def scene_desc(self, sid: int) -> _abi.SceneDesc:
        d = _abi.SceneDesc()
        check(self._lib.mpm_batch_scene_desc(self._h, int(sid), C.byref(d)), "mpm_batch_scene_desc")
        return d

    def tuning(self, interpolation: int, transfer: int) -> dict:
        """Launch settings of the batch's scenes of one (interpolation,
        transfer) combination."""
        t = _abi.Tuning()
        check(self._lib.mpm_batch_get_tuning(self._h, int(interpolation), int(transfer), C.byref(t)),
              "mpm_batch_get_tuning")
        return dict(g2p_chunk=t.g2p_chunk, p2g_stage=t.p2g_stage, p2g_warp_max=t.p2g_warp_max)

    def set_tuning(self, g2p_chunk: int = 1024, p2g_stage: int = 0, interpolation: int = -1, transfer: int = -1,
                   p2g_warp_max: int = -1):
        t = _abi.Tuning(int(g2p_chunk), int(p2g_stage), int(p2g_warp_max))
        check(self._lib.mpm_batch_set_tuning(self._h, int(interpolation), int(transfer), C.byref(t)),
              "mpm_batch_set_tuning")

    def autotune(self, steps_per_candidate: int = 3, force: bool = False, use_disk: bool = True) -> dict:
        """Autotuner over the batch's (stencil, transfer) combinations (see
        MPMSolver3D.autotune); returns the settings per combination present
        and the number of steps taken."""
        flags = (_abi.TUNE_FORCE if force else 0) | (0 if use_disk else _abi.TUNE_NO_DISK)
        run = C.c_int32(0)
        check(self._lib.mpm_batch_autotune(self._h, int(steps_per_candidate), flags, C.byref(run)),
              "mpm_batch_autotune")
        combos = sorted({(self.scene_desc(sid).interpolation, self.scene_desc(sid).transfer) for sid in self._n})
        return {"steps": int(run.value),
                "combinations": [dict(interpolation=i, transfer=t, **self.tuning(i, t)) for i, t in combos]}

    def kernel_spans(self) -> dict:
        """Device-measured time per step (ms) of the P2G, grid and G2P launches
        inside the ordinary graph-replayed steps since the last call, and the
        number of steps: {family: (ms, steps)}."""
        nf = len(_abi.SPAN_FAMILIES)
        ms = (C.c_float * nf)()
        cnt = (C.c_int32 * nf)()
        check(self._lib.mpm_batch_kernel_spans(self._h, ms, cnt, nf), "mpm_batch_kernel_spans")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_abi.SPAN_FAMILIES)}

    def stats(self) -> dict:
        st = _abi.StepStats()
        check(self._lib.mpm_batch_stats(self._h, C.byref(st)), "mpm_batch_stats")
        return dict(active_blocks=st.active_blocks, outside_blocks=st.outside_blocks, active_nodes=st.active_nodes)

    def profile(self, enable: bool = True):
        check(self._lib.mpm_batch_profile(self._h, 1 if enable else 0), "mpm_batch_profile")

    def profile_read(self) -> dict:
        nf = len(_abi.KERNEL_FAMILIES)
        ms = (C.c_float * nf)()
        cnt = (C.c_int32 * nf)()
        check(self._lib.mpm_batch_profile_read(self._h, ms, cnt, nf), "mpm_batch_profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_abi.KERNEL_FAMILIES)}
