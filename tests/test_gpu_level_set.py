"""Level-set collision objects on the GPU against the FP64 oracle: fused step,
split sub-steps, particle collision, both boundary modes, a moving surface;
batch equals solo, checkpoints carry the object, removing it restores the
plain run."""
import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, level_set, scenes
from mpm_b200.batch import Batch
from mpm_b200.level_set import LevelSetCollisionObject3D
from mpm_b200.solver import APICMPMSolver3D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP)


def _scene(transfer, interp, boundary=_abi.BOUNDARY_REFERENCE, n=4000):
    sc = scenes.tiny_scene(n=n, res=24, transfer=transfer, interpolation=interp, boundary=boundary,
                           velocity=(0.5, -20.0, 0.25))
    # obstacle just below the box [0.3, 0.6]^3: its top reaches into the box
    phi = level_set.sphere(sc.origin, sc.resolution, sc.stride, (0.45, 0.2, 0.45), 0.12)
    return sc, phi


def _pair(sc, obj, pcoll=False):
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.set_collision_object(obj)
    o.set_level_set(obj.level_set, obj.friction, obj.velocity)
    if pcoll:
        g.switchIfEnableParticlesCollision()
        o.set_particles_collision(True)
    return g, o


@pytest.mark.parametrize("transfer,interp,boundary,vco,pcoll", [
    (_abi.TRANSFER_APIC, _abi.INTERP_CUBIC, _abi.BOUNDARY_REFERENCE, (0.0, 0.0, 0.0), False),
    (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC, _abi.BOUNDARY_REFERENCE, (0.6, 0.0, -0.3), False),
    (_abi.TRANSFER_APIC, _abi.INTERP_QUADRATIC, _abi.BOUNDARY_STICKY, (0.0, 0.0, 0.0), True),
    (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_LINEAR, _abi.BOUNDARY_REFERENCE, (0.0, 0.2, 0.0), True),
])
def test_fused_step_matches_oracle(gpu, transfer, interp, boundary, vco, pcoll):
    sc, phi = _scene(transfer, interp, boundary)
    obj = LevelSetCollisionObject3D(phi, friction=0.4, velocity=vco)
    g, o = _pair(sc, obj, pcoll)
    g.step(3)
    o.step(3)
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-5, f
    # the obstacle acted: the run differs from the one without it
    free = sc.solver()
    free.step(3)
    assert relerr(free.download(_abi.FIELD_VELOCITY), g.download(_abi.FIELD_VELOCITY)) > 1e-3
    g.close()
    free.close()


@pytest.mark.parametrize("transfer,interp", [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC)])
def test_split_substeps_match_oracle(gpu, transfer, interp):
    sc, phi = _scene(transfer, interp)
    obj = LevelSetCollisionObject3D(phi, friction=0.3, velocity=(0.2, 0.0, 0.0))
    g, o = _pair(sc, obj)
    dt = sc.dt
    g.resetGrid()
    g.particlesToGrid()
    g.computeExternalForces()
    g.updateGridVelocities(dt)
    g.gridCollision(dt)
    if transfer == _abi.TRANSFER_APIC:
        g.gridToParticles(dt)
    else:
        g.gridToParticles(dt, sc.blend)
    g.particlesCollision(dt)
    g.advectParticles(dt)
    o.reset_grid()
    o.particles_to_grid()
    o.gravity()
    o.update_grid_velocities(dt)
    o.grid_collision(dt)
    assert relerr(g.download_grid(_abi.GRID_VELOCITY_STAR), o.grid(_abi.GRID_VELOCITY_STAR)) < 2e-4
    o.grid_to_particles(dt, sc.blend)
    o.particles_collision(dt)
    o.advect(dt)
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-5, f
    g.close()


def test_ball_stays_out_of_the_obstacle(gpu):
    sc, phi = _scene(_abi.TRANSFER_APIC, _abi.INTERP_QUADRATIC, n=20000)
    g = sc.solver()
    g.set_collision_object(LevelSetCollisionObject3D(phi, friction=0.5))
    g.step(400)
    x = g.download(_abi.FIELD_POSITION).astype(np.float64)
    c = np.array([0.45, 0.2, 0.45])
    assert (np.linalg.norm(x - c, axis=1) - 0.12).min() > -sc.stride
    g.close()


def test_batch_equals_solo(gpu):
    scs = scenes.batched_scenes(count=4, scale=0.05)
    objs = []
    for i, s in enumerate(scs):
        phi = level_set.half_space(s.origin, s.resolution, s.stride, (0.0, 0.3 + 0.02 * i, 0.0), (0.2, 1.0, 0.1))
        objs.append(LevelSetCollisionObject3D(phi, friction=0.3 + 0.1 * i, velocity=(0.1 * i, 0.0, 0.0))
                    if i != 2 else None)
    with Batch() as bt:
        ids = [bt.add(s) for s in scs]
        for sid, obj in zip(ids, objs):
            if obj is not None:
                bt.set_collision_object(sid, obj)
        bt.step(20)
        got = [{f: bt.download(sid, f) for f in FIELDS} for sid in ids]
    for s, obj, st in zip(scs, objs, got):
        g = s.solver()
        if obj is not None:
            g.set_collision_object(obj)
        g.step(20)
        for f in FIELDS:
            assert np.array_equal(np.ravel(g.download(f)), np.ravel(st[f])), f
        g.close()


def test_checkpoint_carries_the_object(gpu, tmp_path):
    sc, phi = _scene(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC)
    g = sc.solver()
    g.set_collision_object(LevelSetCollisionObject3D(phi, friction=0.4, velocity=(0.3, 0.0, 0.0)))
    g.step(4)
    path = str(tmp_path / "ls.ckpt")
    g.save(path)
    g.step(6)
    r = APICMPMSolver3D.from_checkpoint(path)
    r.step(6)
    for f in FIELDS:
        assert np.array_equal(g.download(f), r.download(f)), f
    g.close()
    r.close()


def test_removing_the_object(gpu):
    sc, phi = _scene(_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC)
    obj = LevelSetCollisionObject3D(phi, friction=0.4)
    # set and removed before stepping: bitwise the plain run
    a, b = sc.solver(), sc.solver()
    a.set_collision_object(obj)
    a.set_collision_object(None)
    a.step(5)
    b.step(5)
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    # removed between steps (the step graph is already captured): as the oracle
    g, o = _pair(sc, obj)
    g.step(2)
    o.step(2)
    g.set_collision_object(None)
    o.set_level_set(None)
    g.step(3)
    o.step(3)
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-5, f


def test_invalid_level_sets_are_rejected(gpu):
    sc, phi = _scene(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC)
    g = sc.solver()
    bad = phi.copy()
    bad[3, 4, 5] = np.nan
    with pytest.raises(_abi.MPMError):
        g.set_collision_object(LevelSetCollisionObject3D(bad))
    with pytest.raises(_abi.MPMError):
        g.set_collision_object(LevelSetCollisionObject3D(phi, friction=-1.0))
    with pytest.raises(ValueError):
        g.set_collision_object(LevelSetCollisionObject3D(phi[:-1]))
    g.step(1)  # the solver is still usable
    g.close()
