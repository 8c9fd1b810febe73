"""Builder from YAML and the headless C++ driver on the GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

from mpm_b200 import _abi
from mpm_b200.config import buildAPICMPMSolver3DFromYAML, buildMPMSolver3DFromYAML, parseYAML
from mpm_b200.solver import APICMPMSolver3D, Material, MPMSolver3D, Particles

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

YAML = """ParticleGroups:
  - File: a.xyz
    Mass: 0.002
    Velocity: [0.0, -1.0, 0.0]
    YoungModulus: 1.4e5
    PoissonRatio: 0.2
    HardeningCoefficient: 10
    CriticalCompression: 2.5e-2
    CriticalStretch: 7.5e-3
    ConstitutiveModel: FixedCorotated
  - File: b.xyz
    Mass: 0.002
    Velocity: [0.5, 0.0, 0.0]
    YoungModulus: 1.4e5
    PoissonRatio: 0.2
    HardeningCoefficient: 10
    CriticalCompression: 5.0e-2
    CriticalStretch: 9.0e-3
    ConstitutiveModel: FixedCorotated
Grid:
  Origin: [0.0, 0.0, 0.0]
  Resolution: [40, 40, 40]
  Stride: 5e-3
  BoundaryFrictionCoefficient: 0.9
Transfer:
  BlendCoefficient: 0.95
Interpolation:
  Type: CubicBSpline
Simulate:
  deltaTime: 1e-3
Render:
  Offline: false
  ParticleFragmentShader: ../shader/snow.frag
"""


@pytest.fixture()
def scene_dir(tmp_path):
    # integer grid coordinates like the reference's .xyz files, with a
    # half-cell offset group
    rng = np.random.default_rng(3)
    a = np.stack(np.meshgrid(np.arange(12, 20), np.arange(14, 22), np.arange(12, 20), indexing="ij"), -1).reshape(-1, 3)
    b = rng.uniform(22, 28, size=(700, 3))
    (tmp_path / "a.xyz").write_text("\n".join("%d %d %d" % tuple(p) for p in a) + "\n")
    (tmp_path / "b.xyz").write_text("\n".join("%.6f %.6f %.6f" % tuple(p) for p in b) + "\n")
    (tmp_path / "scene.yaml").write_text(YAML)
    return tmp_path


@pytest.mark.parametrize("apic", [False, True])
def test_builder_matches_direct_construction(gpu, scene_dir, apic):
    cfg = parseYAML(str(scene_dir / "scene.yaml"))
    s, n = (buildAPICMPMSolver3DFromYAML if apic else buildMPMSolver3DFromYAML)(cfg)
    assert n == 512 + 700
    # the same particles built by hand, as the reference's builder does
    from mpm_b200.config import readXYZFile
    xa = readXYZFile(str(scene_dir / "a.xyz"), cfg.stride)
    xb = readXYZFile(str(scene_dir / "b.xyz"), cfg.stride)
    mats = [Material(1.4e5, 0.2, 10, 2.5e-2, 7.5e-3), Material(1.4e5, 0.2, 10, 5e-2, 9e-3)]
    p = Particles(np.concatenate([xa, xb]), np.concatenate([np.tile([0, -1, 0], (512, 1)), np.tile([0.5, 0, 0], (700, 1))]),
                  0.002, mats, np.r_[np.zeros(512), np.ones(700)].astype(np.uint16))
    if apic:
        d = APICMPMSolver3D(p, cfg.origin, cfg.resolution, cfg.stride, cfg.friction_coeff, cfg.interp_type,
                            cfg.delta_time)
    else:
        d = MPMSolver3D(p, cfg.origin, cfg.resolution, cfg.stride, cfg.friction_coeff, cfg.blend_coeff,
                        cfg.interp_type, cfg.delta_time)
    s.step(5)
    d.step(5)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE):
        assert np.array_equal(s.download(f), d.download(f))


def test_cli_runs_config(gpu, scene_dir):
    out = scene_dir / "pos.f32"
    r = subprocess.run([os.path.join(ROOT, "mpm_b200", "mpm-run"), str(scene_dir / "scene.yaml"), "--steps", "10",
                        "--apic", "--out", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["particles"] == 1212 and info["steps"] == 10
    pos = np.fromfile(out, np.float32).reshape(-1, 4)
    assert pos.shape == (1212, 4) and np.all(pos[:, 3] == 1) and np.isfinite(pos).all()


def test_cli_implicit_cfl_density(gpu, scene_dir):
    dens = scene_dir / "density.f32"
    r = subprocess.run([os.path.join(ROOT, "mpm_b200", "mpm-run"), str(scene_dir / "scene.yaml"), "--steps", "10",
                        "--apic", "--integration", "implicit", "--max-iter", "30", "--cfl", "0.3",
                        "--density", str(dens)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["particles"] == 1212 and info["steps"] == 10
    # CFL: no step is longer than the configured 1e-3 s
    assert 0 < info["simulated_time"] <= 10 * 1e-3 * (1 + 1e-6)
    d = np.fromfile(dens, np.float32)
    # (a weight at the edge of the cubic stencil can round to -0 ... -1e-16)
    assert d.size == 40 ** 3 and np.isfinite(d).all() and d.min() > -1e-6 * d.max()
    # the density grid integrates to the total particle mass (0.002 per particle)
    assert abs(d.astype(np.float64).sum() * 5e-3 ** 3 / (1212 * 0.002) - 1) < 1e-4
    r = subprocess.run([os.path.join(ROOT, "mpm_b200", "mpm-run"), str(scene_dir / "scene.yaml"), "--integration",
                        "sideways"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
