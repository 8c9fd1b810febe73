"""GPU parity: the sm_100a step against the CPU oracle, through the C ABI.

Tolerances (norm-wise relative, max|gpu - oracle| / max|oracle|) follow the
stated targets: grid mass and momentum 1e-6; particle positions, velocities
and det(Fe)/det(Fp) 1e-5 after one step; forces and B carry the FP32 SVD's
error of the stress and use 1e-4.  Integer work (sorting) is bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from mpm_b200.solver import APICMPMSolver3D, Material, MPMSolver3D, Particles
from oracle import oracle as O

pytestmark = pytest.mark.gpu

COMBOS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2)]  # (transfer, interpolation)


def _sort(keys, bits):
    lib = _abi.load()
    keys = np.ascontiguousarray(keys, np.uint32)
    n = keys.size
    sk = np.empty(n, np.uint32)
    pm = np.empty(n, np.uint32)
    P = C.POINTER(C.c_uint32)
    _abi.check(lib.mpm_sort_keys(keys.ctypes.data_as(P), n, bits, sk.ctypes.data_as(P), pm.ctypes.data_as(P)),
               "mpm_sort_keys")
    return sk, pm


@pytest.mark.parametrize("n,bits,kind", [(1, 8, "rand"), (4095, 12, "rand"), (4097, 22, "dup"),
                                         (100_003, 22, "nearly"), (1_000_000, 24, "dup"), (65536, 32, "rand"),
                                         (50_000, 1, "rand")])
def test_radix_sort_bit_exact(gpu, n, bits, kind):
    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) if bits < 32 else (1 << 32)
    if kind == "rand":
        keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    elif kind == "dup":
        keys = rng.integers(0, 64, n, dtype=np.uint64).astype(np.uint32) * (hi // 64 - 1)
    else:  # nearly sorted with local swaps, like keys between steps
        keys = np.sort(rng.integers(0, hi, n, dtype=np.uint64)).astype(np.uint32)
        idx = rng.integers(0, n - 1, n // 20)
        keys[idx], keys[idx + 1] = keys[idx + 1].copy(), keys[idx].copy()
    sk, pm = _sort(keys, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(pm, order.astype(np.uint32))
    assert np.array_equal(sk, keys[order])


def _nontrivial_state(sc, seed=0, B_scale=5.0):
    rng = np.random.default_rng(seed)
    n = sc.n
    Fe = np.eye(3)[None] + 0.01 * rng.normal(size=(n, 3, 3))
    Fp = np.eye(3)[None] + 0.002 * rng.normal(size=(n, 3, 3))
    B = B_scale * sc.stride ** 2 * rng.normal(size=(n, 3, 3))
    return Fe.astype(np.float32), Fp.astype(np.float32), B.astype(np.float32)


def _pair(sc, seed=0, bits=64):
    """GPU solver and oracle from the same input, with the same non-trivial Fe/Fp/B."""
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=bits)
    Fe, Fp, B = _nontrivial_state(sc, seed)
    for field, val in ((_abi.FIELD_FE, Fe), (_abi.FIELD_FP, Fp)) + (
            ((_abi.FIELD_B, B),) if sc.transfer == _abi.TRANSFER_APIC else ()):
        g.upload(field, val.reshape(sc.n, -1))
        o.set(field, val.reshape(sc.n, -1).astype(np.float64))
    return g, o


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_initial_volume_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=3000, res=24, transfer=transfer, interpolation=interp)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    # V0 = m / (sum_i m_i w_ip / h^3) is a ratio of FP32 sums of up to ~100
    # terms each (about 10 ulp): 3e-6
    assert relerr(g.download(_abi.FIELD_VOLUME0), o.get(_abi.FIELD_VOLUME0)) < 3e-6


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_p2g_grid_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    g, o = _pair(sc)
    g.resetGrid()
    g.particlesToGrid()
    o.reset_grid()
    o.particles_to_grid()
    gm = g.download_grid(_abi.GRID_MASS)
    om = o.grid(_abi.GRID_MASS)
    assert relerr(gm, om) < 1e-6
    # per-node relative error of non-negligible nodes
    big = om > 1e-3 * om.max()
    assert np.abs(gm[big] - om[big]).max() / om[big].min() < 1e-3
    assert np.max(np.abs(gm[big] / om[big] - 1)) < 1e-5
    assert relerr(g.download_grid(_abi.GRID_VELOCITY), o.grid(_abi.GRID_VELOCITY)) < 1e-6
    assert relerr(g.download_grid(_abi.GRID_FORCE), o.grid(_abi.GRID_FORCE)) < 1e-4
    # total mass = total particle mass (partition of unity)
    assert abs(gm.astype(np.float64).sum() / sc.particles.mass.astype(np.float64).sum() - 1) < 1e-5


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_grid_update_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    g, o = _pair(sc, seed=1)
    dt = sc.dt
    for fn in ("resetGrid", "particlesToGrid", "computeExternalForces"):
        getattr(g, fn)()
    g.updateGridVelocities(dt)
    g.gridCollision(dt)
    o.reset_grid()
    o.particles_to_grid()
    o.gravity()
    o.update_grid_velocities(dt)
    o.grid_collision(dt)
    # v = p/m carries no stress but divides the 1e-6 momentum error by light
    # node masses; v* = v + dt f/m inherits the FP32 stress error of f: the
    # stress is 2 mu U diag(s (s - 1)) U^T with s from an FP32 SVD (absolute
    # error ~1e-6), i.e. ~1e-4 relative at the ~1% strains of this scene, and
    # dt f/m at light nodes carries it into v* at up to ~2x that
    assert relerr(g.download_grid(_abi.GRID_VELOCITY), o.grid(_abi.GRID_VELOCITY)) < 1e-5
    assert relerr(g.download_grid(_abi.GRID_VELOCITY_STAR), o.grid(_abi.GRID_VELOCITY_STAR)) < 2e-4


def _particle_fields(transfer):
    f = [_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP, _abi.FIELD_FE, _abi.FIELD_FP]
    return f + ([_abi.FIELD_B] if transfer == _abi.TRANSFER_APIC else [])


TOL = {_abi.FIELD_POSITION: 1e-5, _abi.FIELD_VELOCITY: 1e-5, _abi.FIELD_DET_FE: 1e-5, _abi.FIELD_DET_FP: 1e-5,
       _abi.FIELD_FE: 1e-5, _abi.FIELD_FP: 1e-5, _abi.FIELD_B: 1e-4}


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_split_substeps_match_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    g, o = _pair(sc, seed=2)
    dt = sc.dt
    g.resetGrid()
    g.particlesToGrid()
    g.computeExternalForces()
    g.updateGridVelocities(dt)
    g.gridCollision(dt)
    g.solveLinearSystem(dt)
    if transfer == _abi.TRANSFER_APIC:
        g.gridToParticles(dt)
    else:
        g.gridToParticles(dt, sc.blend)
    g.advectParticles(dt)
    o.reset_grid()
    o.particles_to_grid()
    o.gravity()
    o.update_grid_velocities(dt)
    o.grid_collision(dt)
    o.grid_to_particles(dt, sc.blend)
    o.advect(dt)
    for f in _particle_fields(transfer):
        assert relerr(g.download(f), o.get(f)) < TOL[f], f


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_fused_step_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    g, o = _pair(sc, seed=3)
    g.step(1)
    o.step(1)
    for f in _particle_fields(transfer):
        assert relerr(g.download(f), o.get(f)) < TOL[f], f


@pytest.mark.parametrize("transfer,interp", [(0, 1), (1, 2)])
def test_hundred_steps_bound(gpu, transfer, interp):
    """After 100 steps positions stay within 1e-4 of the FP64 oracle and
    det(Fe), det(Fp) within 1e-3 (chaotic growth of FP32 round-off)."""
    sc = scenes.tiny_scene(n=3000, res=24, transfer=transfer, interpolation=interp)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.step(100)
    o.step(100)
    assert relerr(g.download(_abi.FIELD_POSITION), o.get(_abi.FIELD_POSITION)) < 1e-4
    assert relerr(g.download(_abi.FIELD_VELOCITY), o.get(_abi.FIELD_VELOCITY)) < 1e-2
    assert relerr(g.download(_abi.FIELD_DET_FE), o.get(_abi.FIELD_DET_FE)) < 1e-3
    assert relerr(g.download(_abi.FIELD_DET_FP), o.get(_abi.FIELD_DET_FP)) < 1e-3


@pytest.mark.parametrize("transfer,interp", [(0, 1), (1, 2)])
def test_bitwise_deterministic(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=20000, res=32, transfer=transfer, interpolation=interp)
    a, b = sc.solver(), sc.solver()
    a.step(20)
    b.step(20)
    for f in _particle_fields(transfer):
        assert np.array_equal(a.download(f), b.download(f)), f


def test_reused_streams_and_sorted_upload_deterministic(gpu):
    """Solvers created after others were destroyed run on those engines'
    streams (a per-device cache); a 100k-particle scene is uploaded in
    cell-sorted order.  Every instance steps to the same bits, with
    asynchronous downloads between the steps."""
    n = 100_000
    _, x, v = _shuffled_box(n, 23)
    p = Particles(x, v, 0.0008, [Material(**scenes.SNOW)])

    def run():
        g = APICMPMSolver3D(p, (0, 0, 0), (48, 48, 48), 1 / 48, 0.9, _abi.INTERP_CUBIC, 1e-4)
        out = np.empty((n, 4), np.float32)
        for _ in range(6):
            g.step(1)
            g.download_async(_abi.FIELD_POSITION4, out.ctypes.data)
        g.download_wait()
        res = [g.download(f) for f in _particle_fields(1)]
        g.close()
        return out, res

    first = run()
    live = APICMPMSolver3D(p, (0, 0, 0), (48, 48, 48), 1 / 48, 0.9, _abi.INTERP_CUBIC, 1e-4)
    live.step(2)
    for _ in range(3):
        again = run()
        assert np.array_equal(again[0], first[0])
        for a, b in zip(again[1], first[1]):
            assert np.array_equal(a, b)
    live.close()
    assert np.array_equal(first[0][:, :3], first[1][0])


def test_mass_conserved_exactly(gpu):
    sc = scenes.snow_cube(n=20000)
    g = sc.solver()
    m0 = g.download(_abi.FIELD_MASS)
    g.step(30)
    assert np.array_equal(g.download(_abi.FIELD_MASS), m0)
    assert np.array_equal(m0, sc.particles.mass)


def test_apic_momentum_conserved(gpu):
    sc = scenes.tiny_scene(n=5000, res=32, transfer=1, interpolation=2, gravity=0.0)
    sc.particles.materials[0].youngs_modulus = 0.0
    sc.particles.velocities = np.random.default_rng(9).normal(size=(sc.n, 3)).astype(np.float32)
    sc.particles.mass = np.full(sc.n, 10.0, np.float32)
    g = sc.solver()
    m = g.download(_abi.FIELD_MASS).astype(np.float64)
    p0 = (m[:, None] * g.download(_abi.FIELD_VELOCITY)).sum(0)
    g.step(5)
    p1 = (m[:, None] * g.download(_abi.FIELD_VELOCITY)).sum(0)
    assert np.abs(p1 - p0).max() < 1e-5 * np.abs(p0).max()


def test_particles_collision_toggle_matches_oracle(gpu):
    sc = scenes.tiny_scene(n=2000, res=16, transfer=0, interpolation=1, velocity=(-30.0, 5.0, 0.0))
    sc.particles.positions[:, 0] -= 0.25  # touch the lower x wall
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    assert not g._enable_particles_collision
    g.switchIfEnableParticlesCollision()
    assert g._enable_particles_collision
    o.set_particles_collision(True)
    g.step(3)
    o.step(3)
    assert relerr(g.download(_abi.FIELD_VELOCITY), o.get(_abi.FIELD_VELOCITY)) < 1e-5
    assert relerr(g.download(_abi.FIELD_POSITION), o.get(_abi.FIELD_POSITION)) < 1e-5


@pytest.mark.parametrize("boundary", [_abi.BOUNDARY_REFERENCE, _abi.BOUNDARY_STICKY])
def test_boundary_modes_match_oracle(gpu, boundary):
    sc = scenes.tiny_scene(n=3000, res=16, transfer=1, interpolation=1, boundary=boundary,
                           velocity=(0.0, -40.0, 0.0))
    sc.particles.positions[:, 1] -= 0.22  # near the floor
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.step(2)
    o.step(2)
    assert relerr(g.download(_abi.FIELD_VELOCITY), o.get(_abi.FIELD_VELOCITY)) < 1e-5


def test_neo_hookean_and_two_materials_match_oracle(gpu):
    rng = np.random.default_rng(10)
    n = 3000
    x = (0.3 + 0.3 * rng.random((n, 3))).astype(np.float32)
    mats = [Material(model=_abi.MODEL_NEO_HOOKEAN), Material(critical_compression=5e-2, critical_stretch=9e-3)]
    p = Particles(x, (0.3, -1.0, 0.2), 0.0036, mats, (np.arange(n) % 2).astype(np.uint16))
    g = APICMPMSolver3D(p, (0, 0, 0), (24, 24, 24), 1 / 24, 0.9, _abi.INTERP_CUBIC, 1e-4)
    o = O.OracleSolver(g._desc, p, bits=64)
    g.step(1)
    o.step(1)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP):
        assert relerr(g.download(f), o.get(f)) < 1e-5, f
    g.step(2)
    o.step(2)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP):
        assert relerr(g.download(f), o.get(f)) < 5e-5, f


def _shuffled_box(n, seed):
    rng = np.random.default_rng(seed)
    x = (0.25 + 0.5 * rng.random((n, 3))).astype(np.float32)
    v = rng.normal(scale=0.5, size=(n, 3)).astype(np.float32)
    return rng, x, v


def test_sorted_upload_keeps_the_callers_order(gpu):
    """A scene of >= 65536 particles is written in cell-sorted order at upload;
    before any step every field reads back in the caller's order, exactly."""
    n = 100_000
    rng, x, v = _shuffled_box(n, 21)
    m = (0.001 + 0.001 * rng.random(n)).astype(np.float32)
    vol = (1e-6 + 1e-6 * rng.random(n)).astype(np.float32)
    p = Particles(x, v, m, [Material(**scenes.SNOW)], volume=vol)
    g = APICMPMSolver3D(p, (0, 0, 0), (64, 64, 64), 1 / 64, 0.9, _abi.INTERP_QUADRATIC, 1e-4,
                        volume_mode=_abi.VOLUME_PRESCRIBED)
    assert np.array_equal(g.download(_abi.FIELD_POSITION), x)
    assert np.array_equal(g.download(_abi.FIELD_VELOCITY), v)
    assert np.array_equal(g.download(_abi.FIELD_MASS).reshape(-1), m)
    assert np.array_equal(g.download(_abi.FIELD_VOLUME0).reshape(-1), vol)
    x4 = g.download(_abi.FIELD_POSITION4)
    assert np.array_equal(x4[:, :3], x) and np.all(x4[:, 3] == 1.0)
    fe = g.download(_abi.FIELD_FE).reshape(n, 9)
    assert np.array_equal(fe, np.tile(np.eye(3, dtype=np.float32).reshape(9), (n, 1)))
    w = rng.normal(size=(n, 3)).astype(np.float32)
    g.upload(_abi.FIELD_VELOCITY, w)
    assert np.array_equal(g.download(_abi.FIELD_VELOCITY), w)


def test_sorted_upload_two_materials_match_oracle(gpu):
    """Cell-sorted upload with per-particle material ids (gathered with the
    particles), particles outside the grid, and the FP64 oracle in the
    caller's order.  The oracle's FP32 restatement is off FP64 by 4.8e-6 in
    v after one step and 4.0e-5 after three (det(Fe) 6.5e-6 / 1.6e-5; the
    GPU: 5e-7 / 1.9e-6, its first stress being exactly zero at Fe = I);
    swapping the two materials moves v by 4.5e-3 after three steps."""
    n = 70_000
    rng, x, _ = _shuffled_box(n, 22)
    v = (np.array([0.3, -1.0, 0.2]) + rng.normal(scale=0.05, size=(n, 3))).astype(np.float32)
    x[:8] = np.array([3.0, 0.5, 0.5], np.float32)    # outside: the scene's outside block
    x[8:16] = np.array([0.5, -2.0, 0.5], np.float32)
    mats = [Material(model=_abi.MODEL_NEO_HOOKEAN),
            Material(youngs_modulus=1.4e6, critical_compression=5e-2, critical_stretch=9e-3)]
    mid = rng.integers(0, 2, n).astype(np.uint16)
    p = Particles(x, v, 0.0008, mats, mid)
    g = APICMPMSolver3D(p, (0, 0, 0), (48, 48, 48), 1 / 48, 0.9, _abi.INTERP_CUBIC, 1e-4)
    o = O.OracleSolver(g._desc, p, bits=64)
    g.step(1)
    o.step(1)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP):
        assert relerr(g.download(f), o.get(f)) < 1e-5, f
    g.step(2)
    o.step(2)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP):
        assert relerr(g.download(f), o.get(f)) < 5e-5, f


def test_sorted_upload_nan_reports_numeric_error(gpu):
    sc = scenes.tiny_scene(n=70_000, res=32)
    sc.particles.positions[12345] = np.nan
    with pytest.raises(_abi.MPMError) as e:
        g = sc.solver()
        g.step(1)
        g.synchronize()
    assert e.value.status == 6


def test_particles_outside_the_grid(gpu):
    # stencils that miss the grid contribute nothing (src/mpm_solver3d.cu:259-264)
    sc = scenes.tiny_scene(n=1000, res=16, transfer=0, interpolation=2)
    sc.particles.positions[:10] = np.array([5.0, 5.0, 5.0], np.float32)
    sc.particles.positions[10:20] = np.array([-3.0, 0.5, 0.5], np.float32)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.step(2)
    o.step(2)
    assert relerr(g.download(_abi.FIELD_POSITION), o.get(_abi.FIELD_POSITION)) < 1e-5
    assert relerr(g.download(_abi.FIELD_VELOCITY), o.get(_abi.FIELD_VELOCITY)) < 1e-5


def test_nan_input_reports_numeric_error(gpu):
    # a non-finite input position is reported by the first device pass over the
    # particles (the volume initialization inside the constructor)
    sc = scenes.tiny_scene(n=500, res=16)
    sc.particles.positions[7] = np.nan
    with pytest.raises(_abi.MPMError) as e:
        g = sc.solver()
        g.step(1)
        g.synchronize()
    assert e.value.status == 6


def test_nan_during_run_reports_numeric_error(gpu):
    # a state that turns non-finite mid-run (host-injected NaN velocity) is
    # reported by synchronize() after the step that produced it
    sc = scenes.tiny_scene(n=500, res=16)
    g = sc.solver()
    g.step(2)
    v = g.download(_abi.FIELD_VELOCITY)
    v[11] = np.inf
    g.upload(_abi.FIELD_VELOCITY, v)
    g.step(1)
    with pytest.raises(_abi.MPMError) as e:
        g.synchronize()
    assert e.value.status == 6
    g.synchronize()  # the flag is cleared once reported


def test_empty_scene(gpu):
    p = Particles(np.zeros((0, 3), np.float32), (0, 0, 0), 1.0)
    g = MPMSolver3D(p, (0, 0, 0), (8, 8, 8), 1 / 8, 0.9, 0.95, 1, 1e-4)
    g.step(3)
    g.synchronize()
    assert g.download(_abi.FIELD_POSITION).shape == (0, 3)


def test_position4_and_upload_roundtrip(gpu):
    sc = scenes.tiny_scene(n=777, res=16)
    g = sc.solver()
    g.step(4)
    x = g.download(_abi.FIELD_POSITION)
    x4 = g.download(_abi.FIELD_POSITION4)
    assert np.array_equal(x4[:, :3], x) and np.all(x4[:, 3] == 1.0)
    v = np.random.default_rng(0).normal(size=(sc.n, 3)).astype(np.float32)
    g.upload(_abi.FIELD_VELOCITY, v)
    assert np.array_equal(g.download(_abi.FIELD_VELOCITY), v)


def test_golden_fixtures_on_gpu(gpu):
    """The GPU reproduces the committed FP64 oracle fixtures within tolerance."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.json")
    for case in json.load(open(path))["cases"]:
        if case["bits"] != 64:
            continue
        sc = scenes.tiny_scene(seed=case["seed"], n=case["n"], res=case["res"], transfer=case["transfer"],
                               interpolation=case["interp"])
        g = sc.solver()
        g.step(case["steps"])
        x = g.download(_abi.FIELD_POSITION).reshape(-1)[: len(case["x"])]
        v = g.download(_abi.FIELD_VELOCITY).reshape(-1)[: len(case["v"])]
        assert relerr(x, case["x"]) < 1e-5, case["name"]
        assert relerr(v, case["v"]) < 1e-4, case["name"]


@pytest.mark.parametrize("name", ["snow_cube", "two_balls"])
def test_full_size_configs_properties(gpu, name):
    """Full benchmark sizes: finite state, exact mass, bounded deformation."""
    sc = scenes.snow_cube() if name == "snow_cube" else scenes.two_balls()
    g = sc.solver()
    g.step(10)
    g.synchronize()
    x = g.download(_abi.FIELD_POSITION)
    assert np.isfinite(x).all()
    assert np.array_equal(g.download(_abi.FIELD_MASS), sc.particles.mass)
    dFe = g.download(_abi.FIELD_DET_FE)
    lo = (1 - 2.5e-2) ** 3 * 0.999
    hi = (1 + 7.5e-3) ** 3 * 1.001
    assert dFe.min() >= lo and dFe.max() <= hi


def test_batch_matches_individual_solves_bitwise(gpu):
    """Scenes of different transfers, splines, grids and sizes advanced in one
    batch give bitwise the results of solving each alone."""
    from mpm_b200.batch import Batch
    specs = [dict(seed=21, n=3000, res=24, transfer=1, interpolation=2),
             dict(seed=22, n=1500, res=16, transfer=0, interpolation=1),
             dict(seed=23, n=5000, res=32, transfer=1, interpolation=1),
             dict(seed=24, n=800, res=20, transfer=0, interpolation=2),
             dict(seed=25, n=900, res=12, transfer=0, interpolation=0)]
    scs = [scenes.tiny_scene(**s) for s in specs]
    with Batch() as b:
        ids = [b.add(sc) for sc in scs]
        b.step(7)
        b.synchronize()
        for sc, sid in zip(scs, ids):
            g = sc.solver()
            g.step(7)
            for f in _particle_fields(sc.transfer):
                assert np.array_equal(b.download(sid, f), g.download(f)), (sc.name, f)


def test_batch_add_remove_between_steps(gpu):
    """A scene admitted mid-run and another retired mid-run: the remaining
    scenes are unaffected (bitwise), the new one matches a solo run."""
    from mpm_b200.batch import Batch
    a = scenes.tiny_scene(seed=31, n=2000, res=16, transfer=1, interpolation=2)
    b_ = scenes.tiny_scene(seed=32, n=1200, res=24, transfer=0, interpolation=1)
    c = scenes.tiny_scene(seed=33, n=1700, res=20, transfer=1, interpolation=1)
    with Batch() as b:
        ia, ib = b.add(a), b.add(b_)
        b.step(3)
        b.remove(ib)
        ic = b.add(c)
        b.step(4)
        ga, gc = a.solver(), c.solver()
        ga.step(7)
        gc.step(4)
        assert np.array_equal(b.download(ia, _abi.FIELD_POSITION), ga.download(_abi.FIELD_POSITION))
        assert np.array_equal(b.download(ic, _abi.FIELD_POSITION), gc.download(_abi.FIELD_POSITION))
        assert np.array_equal(b.download(ic, _abi.FIELD_FE), gc.download(_abi.FIELD_FE))


def test_download_async_matches_sync(gpu):
    """Queued asynchronous downloads (more than the two staging buffers, and of
    different sizes) deliver the same bytes as synchronous downloads of the
    same states."""
    import torch
    sc = scenes.snow_cube()
    a, b = sc.solver(), sc.solver()
    fields = [_abi.FIELD_POSITION4, _abi.FIELD_FE, _abi.FIELD_POSITION4, _abi.FIELD_VELOCITY, _abi.FIELD_POSITION4]
    outs, expect = [], []
    for f in fields:
        a.step(1)
        b.step(1)
        comps = _abi.FIELD_COMPONENTS[f]
        buf = torch.full((sc.n, comps), float("nan"), dtype=torch.float32).pin_memory()
        a.download_async(f, buf.data_ptr())
        outs.append(buf)
        expect.append(b.download(f).reshape(sc.n, comps))
    a.download_wait()
    for f, got, ref in zip(fields, outs, expect):
        assert np.array_equal(got.numpy(), ref), f
    a.close()
    b.close()


@pytest.mark.parametrize("transfer,interp", [(1, 2), (0, 1)])
def test_results_do_not_depend_on_the_tuned_settings(gpu, transfer, interp):
    """The settings the autotuner chooses -- particles per G2P work item,
    particles staged per P2G pass, the largest P2G item taken by one warp --
    change only how work is spread over the CTAs, never the order of a sum, so
    every result is bitwise the same."""
    sc = scenes.tiny_scene(n=60000, res=24, transfer=transfer, interpolation=interp)  # ~160 per cell
    runs = []
    for chunk, stage, wmax in ((1024, 0, -1), (256, 16, 0), (4096, 24, 4096), (512, 32, 256)):
        g = sc.solver()
        g.set_tuning(g2p_chunk=chunk, p2g_stage=stage, p2g_warp_max=wmax)
        assert g.tuning() == dict(g2p_chunk=chunk, p2g_stage=stage, p2g_warp_max=wmax)
        g.step(3)
        g.set_tuning(g2p_chunk=4096 if chunk != 4096 else 256, p2g_stage=32, p2g_warp_max=0)  # changed mid-run
        g.step(2)
        runs.append({f: g.download(f) for f in _particle_fields(transfer)})
        g.close()
    for r in runs[1:]:
        for f in _particle_fields(transfer):
            assert np.array_equal(runs[0][f], r[f]), f


@pytest.mark.parametrize("transfer,interp", [(1, 2), (0, 1), (1, 1), (0, 0)])
def test_p2g_by_warps_is_bitwise_p2g_by_ctas(gpu, transfer, interp):
    """P2G items taken by whole warps sum their particles in p2gKernel's
    order, so which kernel takes an item changes no bit: every item by CTAs
    (threshold 0), every item by warps (4096: dense items whose cells hold
    more than one 96-particle segment, segments across staging passes) and
    the engine's own choice agree bitwise, on a dense and on a sparse scene."""
    dense = scenes.tiny_scene(seed=41, n=60000, res=24, transfer=transfer, interpolation=interp)  # ~160 per cell
    sparse = scenes.tiny_scene(seed=42, n=6000, res=32, transfer=transfer, interpolation=interp)  # < 1 per cell
    for sc in (dense, sparse):
        runs = []
        for wmax in (0, 4096, -1):
            g = sc.solver()
            g.set_tuning(p2g_warp_max=wmax)
            g.step(4)
            runs.append({f: g.download(f) for f in _particle_fields(transfer)})
            g.close()
        for r in runs[1:]:
            for f in _particle_fields(transfer):
                assert np.array_equal(runs[0][f], r[f]), (sc.name, f)


def test_p2g_warp_rule_decided_on_the_device(gpu):
    """A sparse scene with thousands of small work items (the engine's rule
    gives them to warps from the first step, decided on the device) against
    every item by CTAs and every item by warps: bitwise the same."""
    sc = scenes.tiny_scene(seed=46, n=20000, res=192, transfer=1, interpolation=2)  # ~3k blocks of ~6
    runs = []
    for wmax in (-1, 0, 4096):
        g = sc.solver()
        g.set_tuning(p2g_warp_max=wmax)
        g.step(3)
        runs.append({f: g.download(f) for f in _particle_fields(1)})
        g.close()
    for r in runs[1:]:
        for f in _particle_fields(1):
            assert np.array_equal(runs[0][f], r[f]), f


def test_p2g_by_warps_in_a_batch(gpu):
    """The same in a batch of two (stencil, transfer) combinations, whose
    P2G lists are kept per combination."""
    from mpm_b200.batch import Batch
    scs = [scenes.tiny_scene(seed=43, n=20000, res=24, transfer=1, interpolation=2),
           scenes.tiny_scene(seed=44, n=3000, res=20, transfer=0, interpolation=1),
           scenes.tiny_scene(seed=45, n=8000, res=28, transfer=1, interpolation=2)]
    runs = []
    for wmax in (0, 4096):
        with Batch() as b:
            ids = [b.add(sc) for sc in scs]
            b.set_tuning(p2g_warp_max=wmax)
            b.step(4)
            runs.append([{f: b.download(sid, f) for f in _particle_fields(sc.transfer)} for sc, sid in zip(scs, ids)])
    for sc, a, c in zip(scs, runs[0], runs[1]):
        for f in a:
            assert np.array_equal(a[f], c[f]), (sc.name, f)


def test_autotune_keeps_results_and_caches(gpu, tmp_path, monkeypatch):
    """The autotuner's steps are ordinary steps (a tuned run equals an untuned
    run of as many steps, bitwise), its choice is one of the candidates, and a
    second solver with the same key takes it from the cache without steps."""
    monkeypatch.setenv("MPM_TUNE_CACHE", str(tmp_path / "tuning.txt"))
    sc = scenes.tiny_scene(n=30000, res=24, transfer=1, interpolation=2)
    a = sc.solver()
    got = a.autotune(steps_per_candidate=1)
    assert got["g2p_chunk"] in (256, 512, 1024, 2048, 4096) and got["p2g_stage"] in (16, 24, 32)
    assert got["p2g_warp_max"] == -1
    assert got["steps"] == 1 + 5 * 2
    a.step(2)
    b = sc.solver()
    b.step(got["steps"] + 2)
    for f in _particle_fields(1):
        assert np.array_equal(a.download(f), b.download(f)), f
    assert (tmp_path / "tuning.txt").read_text().split()[-3:] == [str(got["g2p_chunk"]), str(got["p2g_stage"]),
                                                                  str(got["p2g_warp_max"])]
    c = sc.solver()
    again = c.autotune(steps_per_candidate=1)
    assert again["steps"] == 1 and all(again[k] == got[k] for k in ("g2p_chunk", "p2g_stage", "p2g_warp_max"))


def test_batch_autotune_per_combination(gpu, tmp_path, monkeypatch):
    """In a batch each (stencil, transfer) combination gets its own settings;
    the tuned batch still equals the solo runs bitwise."""
    from mpm_b200.batch import Batch
    monkeypatch.setenv("MPM_TUNE_CACHE", str(tmp_path / "tuning.txt"))
    specs = [dict(seed=41, n=8000, res=24, transfer=1, interpolation=2),
             dict(seed=42, n=6000, res=20, transfer=0, interpolation=1)]
    scs = [scenes.tiny_scene(**s) for s in specs]
    with Batch() as b:
        ids = [b.add(sc) for sc in scs]
        rep = b.autotune(steps_per_candidate=1)
        assert len(rep["combinations"]) == 2 and rep["steps"] == 1 + 5 * 2
        b.step(3)
        for sc, sid in zip(scs, ids):
            g = sc.solver()
            g.step(rep["steps"] + 3)
            for f in _particle_fields(sc.transfer):
                assert np.array_equal(b.download(sid, f), g.download(f)), (sc.name, f)
