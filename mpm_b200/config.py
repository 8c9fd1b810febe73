"""Scene configuration and builders with the reference's names.

parseYAML follows src/mpm3d_parser.cpp:20-71 (MPM3DConfiguration,
include/mpm3d_parser.h:13-37); buildMPMSolver3DFromYAML and
buildAPICMPMSolver3DFromYAML follow src/mpm_solver3d_builder.cu:32-129.  The
YAML is parsed by the library's own reader (include/mpm_b200_config.h), so
Python and C/C++ callers see the same result.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

from . import _abi
from ._abi import check
from .solver import APICMPMSolver3D, Material, MPMSolver3D, Particles


@dataclass
class MPM3DConfiguration:
    group_paths: List[str] = field(default_factory=list)
    velocities: List[Tuple[float, float, float]] = field(default_factory=list)
    masses: List[float] = field(default_factory=list)
    youngs: List[float] = field(default_factory=list)
    poissons: List[float] = field(default_factory=list)
    hardenings: List[float] = field(default_factory=list)
    compressions: List[float] = field(default_factory=list)
    stretches: List[float] = field(default_factory=list)
    constitutive_models: List[int] = field(default_factory=list)
    origin: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    resolution: Tuple[int, int, int] = (0, 0, 0)
    stride: float = 0.0
    friction_coeff: float = 0.0
    blend_coeff: float = 0.0
    interp_type: int = _abi.INTERP_CUBIC
    delta_time: float = 0.0
    offline: bool = False
    particle_frag_shader_path: str = ""
    # schema extensions (optional keys)
    gravity: float = 9.80665
    transfer: int = -1
    boundary: int = _abi.BOUNDARY_REFERENCE
    sticky_cells: int = 3
    base_dir: str = "."


def _from_c(cfg: _abi.Config) -> MPM3DConfiguration:
    out = MPM3DConfiguration()
    for i in range(cfg.ngroups):
        g = cfg.groups[i]
        out.group_paths.append(g.file.decode())
        out.velocities.append(tuple(float(v) for v in g.velocity))
        out.masses.append(float(g.mass))
        out.youngs.append(float(g.material.youngs_modulus))
        out.poissons.append(float(g.material.poisson_ratio))
        out.hardenings.append(float(g.material.hardening))
        out.compressions.append(float(g.material.critical_compression))
        out.stretches.append(float(g.material.critical_stretch))
        out.constitutive_models.append(int(g.material.model))
    out.origin = tuple(float(v) for v in cfg.origin)
    out.resolution = tuple(int(v) for v in cfg.resolution)
    out.stride = float(cfg.stride)
    out.friction_coeff = float(cfg.friction)
    out.blend_coeff = float(cfg.blend)
    out.interp_type = int(cfg.interpolation)
    out.delta_time = float(cfg.dt)
    out.offline = bool(cfg.offline)
    out.particle_frag_shader_path = cfg.particle_frag_shader.decode()
    out.gravity = float(cfg.gravity)
    out.transfer = int(cfg.transfer)
    out.boundary = int(cfg.boundary)
    out.sticky_cells = int(cfg.sticky_cells)
    out.base_dir = cfg.base_dir.decode()
    return out


def parseYAML(filePath: str) -> MPM3DConfiguration:
    lib = _abi.load()
    p = C.POINTER(_abi.Config)()
    check(lib.mpm_config_parse_yaml(filePath.encode(), C.byref(p)), "parseYAML")
    try:
        return _from_c(p.contents)
    finally:
        lib.mpm_config_free(p)


def parseYAMLString(text: str, base_dir: str = ".") -> MPM3DConfiguration:
    lib = _abi.load()
    p = C.POINTER(_abi.Config)()
    check(lib.mpm_config_parse_yaml_string(text.encode(), base_dir.encode(), C.byref(p)), "parseYAML")
    try:
        return _from_c(p.contents)
    finally:
        lib.mpm_config_free(p)


def readXYZFile(filePath: str, stride: float = 1.0, base_dir: str | None = None) -> np.ndarray:
    """Point cloud of an .xyz file scaled by `stride` (the builder's scaling)."""
    lib = _abi.load()
    pts = C.POINTER(C.c_float)()
    n = C.c_size_t()
    check(lib.mpm_read_xyz(filePath.encode(), base_dir.encode() if base_dir else None, float(stride), C.byref(pts),
                           C.byref(n)), "readXYZFile")
    try:
        return np.ctypeslib.as_array(pts, shape=(n.value * 3,)).reshape(-1, 3).copy() if n.value else \
            np.zeros((0, 3), np.float32)
    finally:
        lib.mpm_free(pts)


def build_particles(config: MPM3DConfiguration) -> Particles:
    """Stack the particle groups of a configuration (builder.cu:36-73)."""
    groups = []
    for i, path in enumerate(config.group_paths):
        x = readXYZFile(path, config.stride, config.base_dir)
        mat = Material(config.youngs[i], config.poissons[i], config.hardenings[i], config.compressions[i],
                       config.stretches[i], config.constitutive_models[i])
        groups.append(Particles(x, config.velocities[i], config.masses[i], [mat]))
    return Particles.concat(groups)


def _options(config: MPM3DConfiguration) -> dict:
    return dict(gravity=config.gravity, boundary=config.boundary, sticky_cells=config.sticky_cells)


def buildMPMSolver3DFromYAML(config: MPM3DConfiguration):
    """Returns (solver, particlesNumber) like the reference's builder."""
    p = build_particles(config)
    s = MPMSolver3D(p, config.origin, config.resolution, config.stride, config.friction_coeff, config.blend_coeff,
                    config.interp_type, config.delta_time, **_options(config))
    return s, p.n


def buildAPICMPMSolver3DFromYAML(config: MPM3DConfiguration):
    p = build_particles(config)
    s = APICMPMSolver3D(p, config.origin, config.resolution, config.stride, config.friction_coeff,
                        config.interp_type, config.delta_time, **_options(config))
    return s, p.n
