"""YAML configuration, .xyz loading and the C++ facade (no GPU needed).

The parser follows the reference's parseYAML (src/mpm3d_parser.cpp:20-71);
PyYAML is used here only as an independent reader to cross-check it.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import yaml

from mpm_b200 import _abi
from mpm_b200.config import parseYAML, parseYAMLString, readXYZFile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference's own scene files, copied by tests/golden/reference/vendor.py
REF_CONFIG = os.path.join(ROOT, "tests", "golden", "reference", "config")

SAMPLE = """# snow scene in the reference's schema
ParticleGroups:
  - File: pts_a.xyz   # first group
    Mass: 2.0
    Velocity: [0.0, -1.5, 0.25]
    YoungModulus: 1.4e5
    PoissonRatio: 0.2
    HardeningCoefficient: 10
    CriticalCompression: 2.5e-2
    CriticalStretch: 7.5e-3
    ConstitutiveModel: FixedCorotated
  -   File: "pts b.xyz"
      Mass: 1.0
      Velocity: [1, 2, 3]
      YoungModulus: 5e4
      PoissonRatio: 0.3
      HardeningCoefficient: 5
      CriticalCompression: 0.1e-2
      CriticalStretch: 1.0e-3
      ConstitutiveModel: NeoHookean
Grid:
  Origin: [0.0, 0.0, 0.0]
  Resolution: [16, 20, 24]
  Stride: 5e-3
  BoundaryFrictionCoefficient: 0.9
Transfer:
  BlendCoefficient: 0.95
Interpolation:
  Type: QuadraticBSpline
Simulate:
  deltaTime: 1e-3
Render:
  Offline: false
  ParticleFragmentShader: ../shader/snow.frag
"""


def _check_against_pyyaml(cfg, doc):
    groups = doc["ParticleGroups"]
    assert len(cfg.group_paths) == len(groups)
    models = {"FixedCorotated": 0, "NeoHookean": 1}
    for i, g in enumerate(groups):
        assert cfg.group_paths[i] == g["File"]
        assert cfg.masses[i] == pytest.approx(float(g["Mass"]), rel=1e-7)
        assert cfg.velocities[i] == pytest.approx([float(v) for v in g["Velocity"]], rel=1e-7)
        assert cfg.youngs[i] == pytest.approx(float(g["YoungModulus"]), rel=1e-7)
        assert cfg.poissons[i] == pytest.approx(float(g["PoissonRatio"]), rel=1e-7)
        assert cfg.hardenings[i] == pytest.approx(float(g["HardeningCoefficient"]), rel=1e-7)
        assert cfg.compressions[i] == pytest.approx(float(g["CriticalCompression"]), rel=1e-7)
        assert cfg.stretches[i] == pytest.approx(float(g["CriticalStretch"]), rel=1e-7)
        assert cfg.constitutive_models[i] == models[g["ConstitutiveModel"]]
    grid = doc["Grid"]
    assert cfg.origin == pytest.approx([float(v) for v in grid["Origin"]])
    assert list(cfg.resolution) == [int(v) for v in grid["Resolution"]]
    assert cfg.stride == pytest.approx(float(grid["Stride"]), rel=1e-7)
    assert cfg.friction_coeff == pytest.approx(float(grid["BoundaryFrictionCoefficient"]), rel=1e-7)
    assert cfg.blend_coeff == pytest.approx(float(doc["Transfer"]["BlendCoefficient"]), rel=1e-7)
    interp = {"Linear": 0, "QuadraticBSpline": 1, "CubicBSpline": 2}
    assert cfg.interp_type == interp[doc["Interpolation"]["Type"]]
    assert cfg.delta_time == pytest.approx(float(doc["Simulate"]["deltaTime"]), rel=1e-7)
    assert cfg.offline == bool(doc["Render"]["Offline"])
    assert cfg.particle_frag_shader_path == doc["Render"]["ParticleFragmentShader"]


def test_parse_sample_matches_pyyaml():
    cfg = parseYAMLString(SAMPLE)
    # PyYAML reads "1.4e5" as a string (YAML 1.1); the reference's yaml-cpp reads it as a float
    doc = yaml.safe_load(SAMPLE)
    _check_against_pyyaml(cfg, doc)
    assert cfg.gravity == pytest.approx(9.80665) and cfg.transfer == -1 and cfg.boundary == 0


@pytest.mark.parametrize("name", ["snow_cube.yaml", "snow_two_balls_sparse.yaml", "snow_two_balls.yaml",
                                  "snow_text.yaml", "snow_cylinder_dragon.yaml"])
def test_parse_reference_configs(name):
    path = os.path.join(REF_CONFIG, name)
    cfg = parseYAML(path)
    _check_against_pyyaml(cfg, yaml.safe_load(open(path)))
    assert cfg.base_dir == REF_CONFIG


@pytest.mark.parametrize("bad,status", [
    ("Interpolation:\n  Type: Quintic", 3),
    ("ConstitutiveModel: FixedCorotated", 3),
])
def test_parse_errors(bad, status):
    text = SAMPLE.replace("  Type: QuadraticBSpline", "  Type: Quintic") if "Quintic" in bad else \
        SAMPLE.replace("    ConstitutiveModel: FixedCorotated", "    ConstitutiveModel: Hyperelastic")
    with pytest.raises(_abi.MPMError) as e:
        parseYAMLString(text)
    assert e.value.status == status


def test_missing_key_and_missing_file():
    with pytest.raises(_abi.MPMError) as e:
        parseYAMLString(SAMPLE.replace("  Stride: 5e-3\n", ""))
    assert e.value.status == 3 and "Stride" in str(e.value)
    with pytest.raises(_abi.MPMError) as e:
        parseYAML("/nonexistent/config.yaml")
    assert e.value.status == 2


def test_schema_extensions():
    text = SAMPLE.replace("  deltaTime: 1e-3", "  deltaTime: 1e-3\n  Gravity: 9.8\n  Transfer: APIC")
    text = text.replace("  BoundaryFrictionCoefficient: 0.9", "  BoundaryFrictionCoefficient: 0.9\n"
                        "  Boundary: Sticky\n  StickyCells: 2")
    cfg = parseYAMLString(text)
    assert cfg.gravity == pytest.approx(9.8) and cfg.transfer == 1 and cfg.boundary == 1 and cfg.sticky_cells == 2


def test_read_xyz_scales_by_stride(tmp_path):
    pts = np.array([[89.0, 20.0, 90.0], [100.5, -3.0, 7.25]], np.float32)
    f = tmp_path / "p.xyz"
    f.write_text("\n".join(" ".join(repr(float(v)) for v in p) for p in pts) + "\n\n")
    got = readXYZFile(str(f), 5e-3)
    assert np.array_equal(got, (np.float32(5e-3) * pts).astype(np.float32))
    (tmp_path / "bad.xyz").write_text("1 2 3\n4 five 6\n")
    with pytest.raises(_abi.MPMError) as e:
        readXYZFile(str(tmp_path / "bad.xyz"), 1.0)
    assert e.value.status == 3


def test_read_reference_point_cloud():
    x = readXYZFile("../data/cube_sparse.xyz", 5e-3, base_dir=REF_CONFIG)
    assert x.shape == (11907, 3)
    g = x / np.float32(5e-3)  # the file holds integer grid coordinates
    assert np.abs(g - np.round(g)).max() < 1e-3
    assert np.allclose(g.min(0), [89, 19, 89], atol=1e-3) and np.allclose(g.max(0), [111, 41, 111], atol=1e-3)


def test_reference_two_ball_scene(tmp_path):
    """config/snow_two_balls_sparse.yaml with its two point clouds: two groups
    of different plasticity limits, 6,101 + 56,907 particles on the 200^3
    grid, scaled by the stride."""
    from mpm_b200.config import build_particles
    from ref_scenes import unpack_two_balls
    cfg = parseYAML(unpack_two_balls(str(tmp_path)))
    p = build_particles(cfg)
    assert p.n == 6101 + 56907
    assert cfg.compressions == pytest.approx([5.0e-2, 0.1e-2]) and cfg.stretches == pytest.approx([9.0e-3, 1.0e-3])
    x = np.asarray(p.positions)
    assert x.min() > 0.0 and x.max() < 200 * 5e-3
    v = np.asarray(p.velocities)
    assert np.allclose(v[:6101, 0], 2.5) and np.allclose(v[6101:, 0], -2.5)


def test_cpp_facade_compiles_and_links(tmp_path):
    src = tmp_path / "facade.cpp"
    src.write_text("""
#include "chains/mpm_b200.hpp"
int main(int argc, char**) {
  if (argc < 0) {  // link check only: never executed
    std::vector<chains::MaterialPoint3D> ps = {chains::MaterialPoint3D({0.5f, 0.5f, 0.5f}, {0, 0, 0}, 1.f, 10.f,
        1.4e5f, 0.2f, 2.5e-2f, 7.5e-3f, chains::ConstitutiveModel::FIXED_COROTATED)};
    chains::MPMSolver3D s(ps, {0, 0, 0}, {16, 16, 16}, 1.f / 16, 0.9f, 0.95f,
                          chains::InterpolationType::QUADRATIC_BSPLINE, 1e-4f);
    s.simulateOneStep();
    s.switchIfEnableParticlesCollision();
    chains::LevelSetCollisionObject3D obj;
    obj.level_set.assign(16 * 16 * 16, 1.f);
    obj.friction = 0.3f;
    s.setCollisionObject(obj);
    s.clearCollisionObject();
    s.setCfl(0.4f);
    s.setIntegrationType(chains::IntegrationType::SEMI_IMPLICIT, 20, 1e-5f);
    s.solveLinearSystem(1e-4f);
    std::vector<float> rho = s.density();
    double t = s.simulatedTime();
    (void)rho;
    (void)t;
    int n = 0;
    auto cfg = chains::parseYAML("x.yaml");
    chains::APICMPMSolver3D a = chains::buildAPICMPMSolver3DFromYAML(cfg, n);
    a.gridToParticles(1e-4f);
  }
  return 0;
}
""")
    exe = tmp_path / "facade"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", os.path.join(ROOT, "mpm_b200"), "-lmpm_b200", "-Wl,-rpath," + os.path.join(ROOT, "mpm_b200")],
                   check=True)
    assert subprocess.run([str(exe)]).returncode == 0
