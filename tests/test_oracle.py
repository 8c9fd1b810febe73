"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned to the
mathematics the reference implements: B-spline identities
(src/interpolation3d.cu), the APIC inertia tensor D = k h^2 I
(src/apic_mpm_solver3d.cu:151-157), the 3x3 SVD contract of svd3x3
(src/svd_eigen.cu:7-17), the collision cases of applyBoundaryCollision
(src/collision_object3d.cu:41-48), the stress formulas
(src/material_point3d.cu:110-162) and the plasticity clamp (:53-70); plus
FP32-vs-FP64 agreement of the restated step and the committed golden vectors.
"""
import json
import os

import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KINDS = [(0, 2, 1.0), (1, 3, 1.5), (2, 4, 2.0)]  # (type, stencil, range)


@pytest.mark.parametrize("kind,S,r", KINDS)
@pytest.mark.parametrize("bits", [32, 64])
def test_spline_partition_of_unity_and_gradient(kind, S, r, bits):
    xs = np.random.default_rng(0).random(2000)
    tot = sum(O.spline(bits, kind, xs - k)[0] for k in range(-3, 4))
    dtot = sum(O.spline(bits, kind, xs - k)[1] for k in range(-3, 4))
    tol = 1e-6 if bits == 32 else 1e-14
    assert np.abs(tot - 1).max() < tol
    assert np.abs(dtot).max() < 10 * tol
    # linear reproduction: sum_i N(x - i) (i - x) = 0
    lin = sum(O.spline(bits, kind, xs - k)[0] * (k - xs) for k in range(-3, 4))
    assert np.abs(lin).max() < 10 * tol


@pytest.mark.parametrize("kind,k", [(1, 0.25), (2, 1.0 / 3.0)])
def test_apic_inertia_tensor(kind, k):
    # sum_i N(x - i) (i - x)^2 = k (per axis, cell units) for quadratic/cubic
    xs = np.random.default_rng(1).random(2000)
    second = sum(O.spline(64, kind, xs - j)[0] * (j - xs) ** 2 for j in range(-3, 4))
    assert np.abs(second - k).max() < 1e-13


@pytest.mark.parametrize("kind,S,r", KINDS)
def test_spline_support_and_derivative(kind, S, r):
    x = np.linspace(-3, 3, 6001)
    N, dN = O.spline(64, kind, x)
    assert np.all(N[np.abs(x) >= r] == 0)
    assert np.all(N >= 0)
    # derivative against central differences away from the knots
    eps = 1e-6
    Np, _ = O.spline(64, kind, x + eps)
    Nm, _ = O.spline(64, kind, x - eps)
    fd = (Np - Nm) / (2 * eps)
    knots = np.arange(-2, 2.5, 0.5)
    away = np.min(np.abs(x[:, None] - knots[None, :]), axis=1) > 1e-3
    assert np.abs(fd[away] - dN[away]).max() < 1e-5


def test_spline_fp32_matches_fp64_rounding():
    x = np.random.default_rng(2).uniform(-2.2, 2.2, 5000).astype(np.float32).astype(np.float64)
    for kind, _, _ in KINDS:
        n32, d32 = O.spline(32, kind, x)
        n64, d64 = O.spline(64, kind, x)
        assert np.abs(n32 - n64).max() <= 1.2e-7
        assert np.abs(d32 - d64).max() <= 2.5e-7


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_svd_contract(mode):
    rng = np.random.default_rng(3)
    for i in range(300):
        A = np.eye(3) + 0.1 * rng.normal(size=(3, 3))
        if i % 5 == 0:
            A[:, i % 3] *= -1  # inverted element
        if i % 11 == 0:
            A = rng.normal(size=(3, 3))
        U, s, V = O.svd3(A, mode)
        tol = {0: 5e-5, 1: 5e-5, 2: 1e-13}[mode]
        assert np.abs(U @ np.diag(s) @ V.T - A).max() < tol * max(1, np.abs(A).max())
        assert np.abs(U @ U.T - np.eye(3)).max() < max(tol, 1e-6)
        assert np.abs(V @ V.T - np.eye(3)).max() < max(tol, 1e-6)
        assert abs(np.linalg.det(U) - 1) < 1e-5 and abs(np.linalg.det(V) - 1) < 1e-5
        assert s[0] >= s[1] - 1e-6 and s[1] >= abs(s[2]) - 1e-6
        assert np.sign(s[2]) == np.sign(np.linalg.det(A)) or abs(s[2]) < 1e-6


def test_svd_exact_matches_numpy_singular_values():
    rng = np.random.default_rng(4)
    for _ in range(100):
        A = rng.normal(size=(3, 3))
        _, s, _ = O.svd3(A, 2)
        ref = np.linalg.svd(A, compute_uv=False)
        assert np.allclose(np.abs(s), ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("bits", [32, 64])
def test_collision_cases(bits):
    lo, hi = np.zeros(3), np.ones(3)
    # inside: untouched
    assert np.allclose(O.collision(bits, [0.5] * 3, [1, -2, 3], lo, hi, 0.9), [1, -2, 3])
    # separating at the lower wall (v.n >= eps): untouched
    assert np.allclose(O.collision(bits, [0.0, 0.5, 0.5], [1.0, 0.3, 0.0], lo, hi, 0.9), [1.0, 0.3, 0.0])
    # sticking: |v_t| <= -mu v_n
    assert np.allclose(O.collision(bits, [0.0, 0.5, 0.5], [-1.0, 0.5, 0.0], lo, hi, 0.9), [0, 0, 0])
    # sliding: v_t + mu v_n v_t/|v_t|
    out = O.collision(bits, [0.0, 0.5, 0.5], [-0.5, 2.0, 0.0], lo, hi, 0.9)
    assert np.allclose(out, [0.0, 2.0 - 0.9 * 0.5, 0.0], atol=1e-6)
    # upper wall, normal -1
    out = O.collision(bits, [1.0, 0.5, 0.5], [0.5, 2.0, 0.0], lo, hi, 0.9)
    assert np.allclose(out, [0.0, 2.0 - 0.9 * 0.5, 0.0], atol=1e-6)
    # corner: non-unit normal (1,1,0), v.n = -2
    out = O.collision(bits, [0.0, 0.0, 0.5], [-1.0, -1.0, 5.0], lo, hi, 0.1)
    vt = np.array([-1.0, -1.0, 5.0]) - (-2.0) * np.array([1.0, 1.0, 0.0])
    assert np.allclose(out, vt + 0.1 * (-2.0) * vt / np.linalg.norm(vt), atol=1e-5)


@pytest.mark.parametrize("bits", [32, 64])
def test_fixed_corotated_stress(bits):
    # at F = I the stress vanishes; for F = R S V^T it equals 2mu(F-R)F^T + la(J-1)J I
    out, _ = O.stress(bits, 0, np.eye(3), np.eye(3), 1e4, 2e4, 10.0, 1.0)
    assert np.abs(out).max() < 1e-2
    rng = np.random.default_rng(5)
    F = np.eye(3) + 0.05 * rng.normal(size=(3, 3))
    Fp = np.eye(3) + 0.01 * rng.normal(size=(3, 3))
    mu0, la0, xi, V0 = 5.8e4, 3.9e4, 10.0, 2e-6
    out, _ = O.stress(bits, 0, F, Fp, mu0, la0, xi, V0)
    U, s, Vt = np.linalg.svd(F)
    R = U @ Vt
    f = np.exp(xi * (1 - np.linalg.det(Fp)))  # plasticLame (src/material_point3d.cu:158-162)
    mu, la = mu0 * f, la0 * f
    J = np.linalg.det(F)
    ref = V0 * (2 * mu * (F - R) @ F.T + la * (J - 1) * J * np.eye(3))
    assert relerr(out, ref) < (2e-4 if bits == 32 else 1e-10)


def test_neo_hookean_projects_fe():
    F = np.diag([1.01, 0.99, -0.5])  # inverted: projected to s >= FLT_EPSILON
    out, Fe = O.stress(64, 1, F, np.eye(3), 1.0, 1.0, 0.0, 1.0)
    assert np.linalg.det(Fe) > 0
    s = np.linalg.svd(Fe, compute_uv=False)
    assert s.min() >= np.finfo(np.float32).eps * 0.999


@pytest.mark.parametrize("bits", [32, 64])
def test_plasticity_clamp(bits):
    rng = np.random.default_rng(6)
    tc, ts = 2.5e-2, 7.5e-3
    Fe, Fp = np.eye(3), np.eye(3)
    for _ in range(20):
        g = 50.0 * rng.normal(size=(3, 3))
        Fe1, Fp1 = O.update_deformation(bits, Fe, Fp, g, 1e-3, tc, ts)
        s = np.linalg.svd(Fe1, compute_uv=False)
        assert s.max() <= 1 + ts + 1e-5 and s.min() >= 1 - tc - 1e-5
        # F = Fe Fp is preserved by the clamp
        F = (np.eye(3) + 1e-3 * g) @ Fe @ Fp
        assert relerr(Fe1 @ Fp1, F) < (5e-5 if bits == 32 else 1e-12)
        Fe, Fp = Fe1, Fp1


def _state(sc, o):
    return {f: o.get(f) for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP)}


@pytest.mark.parametrize("transfer,interp", [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2)])
def test_fp32_restatement_tracks_fp64(transfer, interp):
    sc = scenes.tiny_scene(n=800, res=16, transfer=transfer, interpolation=interp)
    o64 = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    o32 = O.OracleSolver(sc.desc(), sc.particles, bits=32)
    o64.step(3)
    o32.step(3)
    assert relerr(o32.get(_abi.FIELD_POSITION), o64.get(_abi.FIELD_POSITION)) < 1e-6
    assert relerr(o32.get(_abi.FIELD_VELOCITY), o64.get(_abi.FIELD_VELOCITY)) < 1e-4
    assert relerr(o32.get(_abi.FIELD_DET_FE), o64.get(_abi.FIELD_DET_FE)) < 1e-5


def test_oracle_scatter_is_thread_count_independent():
    sc = scenes.tiny_scene(n=3000, res=16, transfer=1, interpolation=2)
    a = O.OracleSolver(sc.desc(), sc.particles, bits=32, threads=1)
    b = O.OracleSolver(sc.desc(), sc.particles, bits=32, threads=4)
    a.step(2)
    b.step(2)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_B):
        assert np.array_equal(a.get(f), b.get(f))


def test_oracle_grid_mass_is_particle_mass():
    sc = scenes.tiny_scene(n=1000, res=16, transfer=0, interpolation=1)
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    o.reset_grid()
    o.particles_to_grid()
    assert abs(o.grid(_abi.GRID_MASS).sum() - sc.particles.mass.astype(np.float64).sum()) < 1e-12


def test_oracle_apic_conserves_momentum_without_forces():
    # zero stiffness, zero gravity, particles away from the walls: APIC P2G/G2P
    # conserves linear momentum exactly (up to round-off)
    sc = scenes.tiny_scene(n=1500, res=24, transfer=1, interpolation=2, gravity=0.0)
    for m in sc.particles.materials:
        m.youngs_modulus = 0.0
    rng = np.random.default_rng(8)
    sc.particles.velocities = rng.normal(size=(sc.n, 3)).astype(np.float32)
    # Heavy particles: the reference zeroes v* on nodes with mass <= FLT_EPSILON
    # (src/grid3d.cu:37), which would otherwise drop the momentum of far
    # stencil tails.
    sc.particles.mass = np.full(sc.n, 10.0, np.float32)
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    m = o.get(_abi.FIELD_MASS)
    p0 = (m[:, None] * o.get(_abi.FIELD_VELOCITY)).sum(0)
    o.step(3)
    p1 = (m[:, None] * o.get(_abi.FIELD_VELOCITY)).sum(0)
    # exact up to the FLT_EPSILON node-mass cut of the reference (~1e-9 here)
    assert np.abs(p1 - p0).max() < 1e-8 * max(1.0, np.abs(p0).max())


def test_golden_vectors():
    """Committed oracle outputs (tests/golden/make_golden.py) still reproduce."""
    path = os.path.join(GOLDEN, "oracle_golden.json")
    g = json.load(open(path))
    for case in g["cases"]:
        sc = scenes.tiny_scene(seed=case["seed"], n=case["n"], res=case["res"], transfer=case["transfer"],
                               interpolation=case["interp"])
        o = O.OracleSolver(sc.desc(), sc.particles, bits=case["bits"])
        o.step(case["steps"])
        for key, field in (("x", _abi.FIELD_POSITION), ("v", _abi.FIELD_VELOCITY), ("detFe", _abi.FIELD_DET_FE)):
            got = np.asarray(o.get(field)).reshape(-1)[: len(case[key])]
            assert np.allclose(got, case[key], rtol=0, atol=1e-12 if case["bits"] == 64 else 1e-6), (case["name"], key)
