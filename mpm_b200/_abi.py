"""ctypes binding of the C ABI in include/mpm_b200.h and include/mpm_b200_batch.h.

The shared library is built in-tree (``mpm_b200/libmpm_b200.so``).  There is
no CPU fallback: if the library is missing or no CUDA device is visible, the
solver classes raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpm_b200.so")

# ---- enums (mirroring include/mpm_b200.h) ---------------------------------
MPM_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "IO", 3: "PARSE", 4: "OOM", 5: "CUDA", 6: "NUMERIC",
                7: "BUDGET", 8: "TIMEOUT", 9: "UNSUPPORTED"}

INTERP_LINEAR, INTERP_QUADRATIC, INTERP_CUBIC = 0, 1, 2
MODEL_FIXED_COROTATED, MODEL_NEO_HOOKEAN = 0, 1
TRANSFER_PIC_FLIP, TRANSFER_APIC = 0, 1
BOUNDARY_REFERENCE, BOUNDARY_STICKY = 0, 1
VOLUME_GRID_ESTIMATE, VOLUME_PRESCRIBED = 0, 1

FIELD_POSITION, FIELD_VELOCITY, FIELD_FE, FIELD_FP, FIELD_B = 0, 1, 2, 3, 4
FIELD_VOLUME0, FIELD_MASS, FIELD_POSITION4, FIELD_DET_FE, FIELD_DET_FP = 5, 6, 7, 8, 9
FIELD_COMPONENTS = {0: 3, 1: 3, 2: 9, 3: 9, 4: 9, 5: 1, 6: 1, 7: 4, 8: 1, 9: 1}

GRID_MASS, GRID_VELOCITY, GRID_FORCE, GRID_VELOCITY_STAR = 0, 1, 2, 3
GRID_COMPONENTS = {0: 1, 1: 3, 2: 3, 3: 3}

# kernel families of mpm_solver_kernel_spans (device-measured inside the step)
SPAN_FAMILIES = ["p2g", "grid", "g2p"]
# kernel families reported by mpm_solver_profile_read
KERNEL_FAMILIES = ["keys", "sort", "compact", "stress", "p2g", "grid", "g2p"]


# autotuner flags (mpm_solver_autotune)
TUNE_FORCE, TUNE_NO_DISK = 1, 2
G2P_CHUNK_MIN, G2P_CHUNK_MAX = 256, 4096
P2G_WARP_MAX_MAX = 4096


class Tuning(C.Structure):
    _fields_ = [("g2p_chunk", C.c_int32), ("p2g_stage", C.c_int32), ("p2g_warp_max", C.c_int32)]


class Material(C.Structure):
    _fields_ = [("youngs_modulus", C.c_float), ("poisson_ratio", C.c_float), ("hardening", C.c_float),
                ("critical_compression", C.c_float), ("critical_stretch", C.c_float), ("model", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("resolution", C.c_int32 * 3), ("stride", C.c_float),
                ("friction", C.c_float), ("blend", C.c_float), ("dt", C.c_float), ("gravity", C.c_float),
                ("transfer", C.c_int32), ("interpolation", C.c_int32), ("boundary", C.c_int32),
                ("sticky_cells", C.c_int32), ("volume_mode", C.c_int32), ("particles_collision", C.c_int32)]


class ParticlesIn(C.Structure):
    _fields_ = [("n", C.c_size_t), ("position", C.POINTER(C.c_float)), ("velocity", C.POINTER(C.c_float)),
                ("mass", C.POINTER(C.c_float)), ("material", C.POINTER(C.c_uint16)),
                ("volume", C.POINTER(C.c_float)), ("materials", C.POINTER(Material)), ("nmaterials", C.c_int32)]


class ConfigGroup(C.Structure):
    _fields_ = [("file", C.c_char * 1024), ("mass", C.c_float), ("velocity", C.c_float * 3),
                ("material", Material)]


class Config(C.Structure):
    _fields_ = [("ngroups", C.c_int32), ("groups", C.POINTER(ConfigGroup)), ("origin", C.c_float * 3),
                ("resolution", C.c_int32 * 3), ("stride", C.c_float), ("friction", C.c_float), ("blend", C.c_float),
                ("interpolation", C.c_int32), ("dt", C.c_float), ("offline", C.c_int32),
                ("particle_frag_shader", C.c_char * 1024), ("gravity", C.c_float), ("transfer", C.c_int32),
                ("boundary", C.c_int32), ("sticky_cells", C.c_int32), ("base_dir", C.c_char * 1024)]


class StepStats(C.Structure):
    _fields_ = [("active_blocks", C.c_uint32), ("outside_blocks", C.c_uint32), ("active_nodes", C.c_uint32),
                ("reserved", C.c_uint32)]


# Every exported entry point: name -> (restype, argtypes)
_P = C.c_void_p
_F = C.POINTER(C.c_float)
SIGNATURES = {
    "mpm_abi_version": (C.c_int32, []),
    "mpm_last_error_string": (C.c_char_p, []),
    "mpm_device_count": (C.c_int, [C.POINTER(C.c_int32)]),
    "mpm_solver_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(ParticlesIn), C.POINTER(_P)]),
    "mpm_solver_destroy": (C.c_int, [_P]),
    "mpm_solver_save": (C.c_int, [_P, C.c_char_p]),
    "mpm_solver_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mpm_solver_step": (C.c_int, [_P, C.c_int32]),
    "mpm_solver_synchronize": (C.c_int, [_P]),
    "mpm_solver_initialize": (C.c_int, [_P]),
    "mpm_solver_reset_grid": (C.c_int, [_P]),
    "mpm_solver_particles_to_grid": (C.c_int, [_P]),
    "mpm_solver_compute_external_forces": (C.c_int, [_P]),
    "mpm_solver_compute_gravity_forces": (C.c_int, [_P]),
    "mpm_solver_update_grid_velocities": (C.c_int, [_P, C.c_float]),
    "mpm_solver_grid_collision": (C.c_int, [_P, C.c_float]),
    "mpm_solver_solve_linear_system": (C.c_int, [_P, C.c_float]),
    "mpm_solver_grid_to_particles": (C.c_int, [_P, C.c_float, C.c_float]),
    "mpm_solver_particles_collision": (C.c_int, [_P, C.c_float]),
    "mpm_solver_advect_particles": (C.c_int, [_P, C.c_float]),
    "mpm_solver_set_particles_collision": (C.c_int, [_P, C.c_int32]),
    "mpm_solver_get_particles_collision": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "mpm_solver_num_particles": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "mpm_solver_get_desc": (C.c_int, [_P, C.POINTER(SceneDesc)]),
    "mpm_solver_download": (C.c_int, [_P, C.c_int32, _F]),
    "mpm_solver_download_async": (C.c_int, [_P, C.c_int32, C.c_void_p]),
    "mpm_solver_download_wait": (C.c_int, [_P]),
    "mpm_solver_download_density": (C.c_int, [_P, _F]),
    "mpm_solver_set_level_set": (C.c_int, [_P, _F, C.c_float, _F]),
    "mpm_solver_set_cfl": (C.c_int, [_P, C.c_float]),
    "mpm_solver_set_implicit": (C.c_int, [_P, C.c_float, C.c_int32, C.c_float]),
    "mpm_solver_solve_info": (C.c_int, [_P, C.POINTER(C.c_int32), _F]),
    "mpm_solver_time": (C.c_int, [_P, C.POINTER(C.c_double), _F]),
    "mpm_solver_download_grid": (C.c_int, [_P, C.c_int32, _F]),
    "mpm_solver_upload": (C.c_int, [_P, C.c_int32, _F]),
    "mpm_solver_profile": (C.c_int, [_P, C.c_int32]),
    "mpm_solver_profile_read": (C.c_int, [_P, _F, C.POINTER(C.c_int32), C.c_int32]),
    "mpm_sort_keys": (C.c_int, [C.POINTER(C.c_uint32), C.c_size_t, C.c_int32, C.POINTER(C.c_uint32),
                                C.POINTER(C.c_uint32)]),
    "mpm_sort_keys_device_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p, C.c_void_p,
                                               C.c_void_p]),
    "mpm_set_device": (C.c_int, [C.c_int32]),
    "mpm_release_cached_memory": (C.c_int, [C.c_int32]),
    "mpm_config_parse_yaml": (C.c_int, [C.c_char_p, C.POINTER(C.POINTER(Config))]),
    "mpm_config_parse_yaml_string": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.POINTER(Config))]),
    "mpm_config_free": (C.c_int, [C.POINTER(Config)]),
    "mpm_read_xyz": (C.c_int, [C.c_char_p, C.c_char_p, C.c_float, C.POINTER(C.POINTER(C.c_float)),
                               C.POINTER(C.c_size_t)]),
    "mpm_free": (None, [C.c_void_p]),
    "mpm_solver_create_from_config": (C.c_int, [C.POINTER(Config), C.c_int32, C.POINTER(_P), C.POINTER(C.c_int32)]),
    "mpm_solver_stats": (C.c_int, [_P, C.POINTER(StepStats)]),
    "mpm_batch_stats": (C.c_int, [_P, C.POINTER(StepStats)]),
    "mpm_solver_write_vdb": (C.c_int, [_P, C.c_char_p]),
    "mpm_batch_write_vdb": (C.c_int, [_P, C.c_int32, C.c_char_p]),
    "mpm_batch_time_steps": (C.c_int, [_P, C.c_int32]),
    "mpm_solver_kernel_spans": (C.c_int, [_P, _F, C.POINTER(C.c_int32), C.c_int32]),
    "mpm_batch_kernel_spans": (C.c_int, [_P, _F, C.POINTER(C.c_int32), C.c_int32]),
    "mpm_batch_step_times": (C.c_int, [_P, _F, C.c_int32, C.POINTER(C.c_int32)]),
    "mpm_batch_wait_steps": (C.c_int, [_P, C.c_int32]),
    "mpm_write_vdb_density": (C.c_int, [_F, C.POINTER(C.c_int32), C.c_char_p]),
    "mpm_solver_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "mpm_solver_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "mpm_solver_autotune": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "mpm_batch_get_tuning": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(Tuning)]),
    "mpm_batch_set_tuning": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(Tuning)]),
    "mpm_batch_autotune": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "mpm_solver_timed_step": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float)]),
    "mpm_kernel_launches": (C.c_int, [C.POINTER(C.c_uint64)]),
    "mpm_batch_timed_step": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float)]),
    "mpm_batch_create": (C.c_int, [C.POINTER(_P)]),
    "mpm_batch_destroy": (C.c_int, [_P]),
    "mpm_batch_add_scene": (C.c_int, [_P, C.POINTER(SceneDesc), C.POINTER(ParticlesIn), C.POINTER(C.c_int32)]),
    "mpm_batch_remove_scene": (C.c_int, [_P, C.c_int32]),
    "mpm_batch_save_scene": (C.c_int, [_P, C.c_int32, C.c_char_p]),
    "mpm_batch_load_scene": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int32)]),
    "mpm_batch_step": (C.c_int, [_P, C.c_int32]),
    "mpm_batch_synchronize": (C.c_int, [_P]),
    "mpm_batch_download": (C.c_int, [_P, C.c_int32, C.c_int32, _F]),
    "mpm_batch_download_async": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_void_p]),
    "mpm_batch_download_wait": (C.c_int, [_P]),
    "mpm_batch_download_density": (C.c_int, [_P, C.c_int32, _F]),
    "mpm_batch_set_level_set": (C.c_int, [_P, C.c_int32, _F, C.c_float, _F]),
    "mpm_batch_set_cfl": (C.c_int, [_P, C.c_int32, C.c_float]),
    "mpm_batch_set_implicit": (C.c_int, [_P, C.c_int32, C.c_float, C.c_int32, C.c_float]),
    "mpm_batch_solve_info": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), _F]),
    "mpm_batch_time": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_double), _F]),
    "mpm_batch_num_scenes": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "mpm_batch_scene_particles": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_size_t)]),
    "mpm_batch_scene_desc": (C.c_int, [_P, C.c_int32, C.POINTER(SceneDesc)]),
    "mpm_batch_profile": (C.c_int, [_P, C.c_int32]),
    "mpm_batch_profile_read": (C.c_int, [_P, _F, C.POINTER(C.c_int32), C.c_int32]),
}


class MPMError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")


_lib = None


def load() -> C.CDLL:
    """Load libmpm_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing; run `python mpm_b200/build.py` (needs nvcc)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != MPM_OK:
        msg = load().mpm_last_error_string()
        raise MPMError(status, where, msg.decode() if msg else "")


def device_count() -> int:
    n = C.c_int32(0)
    load().mpm_device_count(C.byref(n))
    return int(n.value)
