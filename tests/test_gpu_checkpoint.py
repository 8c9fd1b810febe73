"""Checkpoint and resume: a solver (or batch scene) restored from a checkpoint
takes bitwise the steps the saved one takes."""
import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from mpm_b200.batch import Batch
from mpm_b200.solver import APICMPMSolver3D, MPMSolver3D

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP, _abi.FIELD_VOLUME0)


def _state(get, apic):
    fs = FIELDS + ((_abi.FIELD_B,) if apic else ())
    return {f: np.array(get(f)) for f in fs}


def _same(a, b):
    for f in a:
        assert np.array_equal(np.ravel(a[f]), np.ravel(b[f])), f


@pytest.mark.parametrize("transfer,interp", [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC)])
def test_solver_resume_is_bitwise(gpu, tmp_path, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    apic = transfer == _abi.TRANSFER_APIC
    g = sc.solver()
    g.step(5)
    g.switchIfEnableParticlesCollision()  # part of the saved description
    path = str(tmp_path / "s.ckpt")
    g.save(path)
    g.step(6)
    ref = _state(g.download, apic)
    cls = APICMPMSolver3D if apic else MPMSolver3D
    r = cls.from_checkpoint(path)
    assert r._enable_particles_collision
    r.step(6)
    _same(_state(r.download, apic), ref)
    g.close()
    r.close()


def test_checkpoint_right_after_construction(gpu, tmp_path):
    sc = scenes.tiny_scene(n=3000, res=16)
    g = sc.solver()
    path = str(tmp_path / "c.ckpt")
    g.save(path)
    g.step(4)
    r = APICMPMSolver3D.from_checkpoint(path)
    r.step(4)
    _same(_state(r.download, True), _state(g.download, True))


def test_batch_scene_resume_is_bitwise(gpu, tmp_path):
    scs = scenes.batched_scenes(count=3, scale=0.02)
    with Batch() as b:
        ids = [b.add(s) for s in scs]
        b.step(3)
        path = str(tmp_path / "b.ckpt")
        b.save_scene(ids[1], path)
        b.step(4)
        apic = scs[1].transfer == _abi.TRANSFER_APIC
        ref = _state(lambda f: b.download(ids[1], f), apic)
    # into a fresh batch beside another scene, and into a plain solver
    with Batch() as b2:
        other = b2.add(scs[0])
        sid = b2.load_scene(path)
        assert sid != other
        b2.step(4)
        _same(_state(lambda f: b2.download(sid, f), apic), ref)
    cls = APICMPMSolver3D if apic else MPMSolver3D
    r = cls.from_checkpoint(path)
    r.step(4)
    _same(_state(r.download, apic), ref)
    r.close()
