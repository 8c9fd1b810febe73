"""Semi-implicit update on the GPU (the reference's solveLinearSystem is a
TODO, src/mpm_solver3d.cu:312-314): the FP32 conjugate-residual solve against
the FP64 oracle solved to 1e-12, fused implicit steps against the oracle's,
bitwise determinism, batch equals solo, checkpoints carry the settings."""
import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from mpm_b200.batch import Batch
from mpm_b200.solver import APICMPMSolver3D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP)


def _pair(transfer, interp, model=_abi.MODEL_FIXED_COROTATED, n=4000, seed=5, dt=None):
    sc = scenes.tiny_scene(n=n, res=24, transfer=transfer, interpolation=interp, velocity=(0.5, -3.0, 0.25))
    sc.particles.materials[0].model = model
    if dt:
        sc.dt = dt
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    rng = np.random.default_rng(seed)
    Fe = (np.eye(3)[None] + 0.03 * rng.normal(size=(sc.n, 3, 3))).astype(np.float32)
    Fp = (np.eye(3)[None] + 0.005 * rng.normal(size=(sc.n, 3, 3))).astype(np.float32)
    for f, v in ((_abi.FIELD_FE, Fe), (_abi.FIELD_FP, Fp)):
        g.upload(f, v.reshape(sc.n, 9))
        o.set(f, v.reshape(sc.n, 9).astype(np.float64))
    return sc, g, o


@pytest.mark.parametrize("transfer,interp,model", [
    (_abi.TRANSFER_APIC, _abi.INTERP_CUBIC, _abi.MODEL_FIXED_COROTATED),
    (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC, _abi.MODEL_FIXED_COROTATED),
    (_abi.TRANSFER_APIC, _abi.INTERP_QUADRATIC, _abi.MODEL_NEO_HOOKEAN),
])
def test_split_solve_matches_oracle(gpu, transfer, interp, model):
    sc, g, o = _pair(transfer, interp, model)
    dt = 1e-3  # 10x the scene's explicit step
    g.set_implicit(1.0, max_iter=200, tol=1e-6)
    o.set_implicit(1.0, max_iter=500, tol=1e-12)
    g.resetGrid()
    g.particlesToGrid()
    g.computeExternalForces()
    g.updateGridVelocities(dt)
    g.gridCollision(dt)
    vs0 = g.download_grid(_abi.GRID_VELOCITY_STAR)
    g.solveLinearSystem(dt)
    o.reset_grid()
    o.particles_to_grid()
    o.gravity()
    o.update_grid_velocities(dt)
    o.grid_collision(dt)
    o.solve_linear_system(dt)
    it, res = g.solve_info()
    assert 0 < it < 200 and res <= 1e-6, (it, res)
    got, ref = g.download_grid(_abi.GRID_VELOCITY_STAR), o.grid(_abi.GRID_VELOCITY_STAR)
    assert relerr(got, ref) < 1e-4
    assert relerr(vs0, ref) > 1e-3  # the solve changed v*


@pytest.mark.parametrize("transfer,interp", [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC)])
def test_implicit_steps_match_oracle(gpu, transfer, interp):
    sc, g, o = _pair(transfer, interp, dt=5e-4)
    g.set_implicit(1.0, max_iter=200, tol=1e-6)
    o.set_implicit(1.0, max_iter=500, tol=1e-12)
    g.step(4)
    o.step(4)
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-4, f
    it, res = g.solve_info()
    assert it > 0 and res <= 1e-6


def test_implicit_is_bitwise_deterministic(gpu):
    sc = scenes.tiny_scene(n=20000, res=32, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC)
    sc.dt = 1e-3  # the solves iterate
    a, b = sc.solver(), sc.solver()
    for s in (a, b):
        s.set_implicit(0.5, max_iter=40, tol=1e-6)
        s.step(8)
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    assert a.solve_info() == b.solve_info()
    assert a.solve_info()[0] > 0


def test_batch_with_implicit_scenes_equals_solo(gpu):
    scs = scenes.batched_scenes(count=4, scale=0.05)
    scs[0].dt = scs[2].dt = 1e-3  # the solves iterate
    betas = [1.0, 0.0, 0.5, 0.0]
    with Batch() as bt:
        ids = [bt.add(s) for s in scs]
        for sid, beta in zip(ids, betas):
            if beta:
                bt.set_implicit(sid, beta, max_iter=30, tol=1e-6)
        bt.step(6)
        got = [{f: bt.download(sid, f) for f in FIELDS} for sid in ids]
        info = [bt.solve_info(sid) for sid in ids]
    for s, beta, st, inf in zip(scs, betas, got, info):
        g = s.solver()
        if beta:
            g.set_implicit(beta, max_iter=30, tol=1e-6)
        g.step(6)
        for f in FIELDS:
            assert np.array_equal(np.ravel(g.download(f)), np.ravel(st[f])), f
        if beta:
            assert g.solve_info() == inf
            assert inf[0] > 0
        g.close()


def test_checkpoint_carries_the_settings(gpu, tmp_path):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_CUBIC)
    g = sc.solver()
    g.set_implicit(1.0, max_iter=25, tol=1e-6)
    g.step(3)
    path = str(tmp_path / "imp.ckpt")
    g.save(path)
    g.step(4)
    r = APICMPMSolver3D.from_checkpoint(path)
    r.step(4)
    for f in FIELDS:
        assert np.array_equal(g.download(f), r.download(f)), f


def test_back_to_explicit(gpu):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=_abi.TRANSFER_PIC_FLIP, interpolation=_abi.INTERP_QUADRATIC)
    a, b = sc.solver(), sc.solver()
    a.set_implicit(1.0)
    a.set_implicit(0.0)
    a.step(5)
    b.step(5)
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f


def test_stiff_block_at_large_dt(gpu):
    """The stiff block that blows up explicitly (tests/test_implicit.py) stays
    bounded with beta = 1 and follows the oracle's implicit run."""
    from test_implicit import jelly
    sc = jelly(n=2000)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.set_implicit(1.0, max_iter=100, tol=1e-6)
    o.set_implicit(1.0, max_iter=200, tol=1e-10)
    g.step(20)
    o.step(20)
    v = g.download(_abi.FIELD_VELOCITY)
    assert np.isfinite(v).all() and np.abs(v).max() < 0.5
    assert relerr(g.download(_abi.FIELD_POSITION), o.get(_abi.FIELD_POSITION)) < 1e-4
    assert relerr(v, o.get(_abi.FIELD_VELOCITY)) < 1e-2


def test_graphed_and_direct_solves_agree_at_the_iteration_cap(gpu, monkeypatch):
    """With tol = 0 every solve runs to max_iter.  Replayed from the step
    graph the iterations are a conditional while node; with graphs off
    (MPM_NO_GRAPHS, read when a solver is created) they are max_iter direct
    launches of the same kernels.  Both give bitwise the same state and the
    same iteration count and residual."""
    sc = scenes.tiny_scene(n=6000, res=24, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC)
    sc.dt = 1e-3
    graphed = sc.solver()
    monkeypatch.setenv("MPM_NO_GRAPHS", "1")
    direct = sc.solver()
    monkeypatch.delenv("MPM_NO_GRAPHS")
    for s in (graphed, direct):
        s.set_implicit(1.0, max_iter=12, tol=0.0)
        s.step(6)
    for f in FIELDS:
        assert np.array_equal(graphed.download(f), direct.download(f)), f
    assert graphed.solve_info() == direct.solve_info()
    assert graphed.solve_info()[0] == 12
