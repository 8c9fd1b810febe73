"""CFL time step on the GPU against the FP64 oracle: the step's dt comes from
the device-side max |v_p| (no host round trip), the simulated time and the
last dt match, batches equal solo runs, checkpoints carry both."""
import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from mpm_b200.batch import Batch
from mpm_b200.solver import APICMPMSolver3D, MPMSolver3D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP)


def _fast(transfer, interp):
    return scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp, velocity=(0.5, -30.0, 0.25))


@pytest.mark.parametrize("transfer,interp", [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC)])
def test_cfl_steps_match_oracle(gpu, transfer, interp):
    sc = _fast(transfer, interp)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.set_cfl(0.08)
    o.set_cfl(0.08)
    for _ in range(3):  # the first steps run directly, later ones replay the step graph
        g.step(2)
        o.step(2)
        tg, dg = g.time()
        to, do = o.time()
        assert dg < sc.dt
        # dt from FP32 velocities that carry the step tolerance
        assert abs(dg / do - 1) < 1e-5
        assert abs(tg / to - 1) < 1e-5
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-5, f
    g.close()


def test_switching_cfl_off_restores_the_fixed_dt(gpu):
    sc = _fast(_abi.TRANSFER_APIC, _abi.INTERP_QUADRATIC)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.set_cfl(0.05)
    o.set_cfl(0.05)
    g.step(3)
    o.step(3)
    g.set_cfl(0.0)
    o.set_cfl(0.0)
    g.step(3)
    o.step(3)
    t, dt = g.time()
    assert dt == np.float32(sc.dt)
    assert abs(t / o.time()[0] - 1) < 1e-5
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-5, f


def test_scene_at_rest_keeps_the_fixed_dt(gpu):
    sc = scenes.tiny_scene(n=2000, res=16, gravity=0.0, velocity=(0.0, 0.0, 0.0))
    g = sc.solver()
    g.set_cfl(0.3)
    g.step(4)
    t, dt = g.time()
    assert dt == np.float32(sc.dt)
    assert abs(t - 4 * float(np.float32(sc.dt))) < 1e-12


def test_batch_with_mixed_cfl_equals_solo(gpu):
    scs = scenes.batched_scenes(count=4, scale=0.05)
    cfls = [0.05, 0.0, 0.2, 0.0]
    with Batch() as bt:
        ids = [bt.add(s) for s in scs]
        for sid, c in zip(ids, cfls):
            if c:
                bt.set_cfl(sid, c)
        bt.step(12)
        got = [({f: bt.download(sid, f) for f in FIELDS}, bt.time(sid)) for sid in ids]
    for s, c, (st, tm) in zip(scs, cfls, got):
        g = s.solver()
        if c:
            g.set_cfl(c)
        g.step(12)
        for f in FIELDS:
            assert np.array_equal(np.ravel(g.download(f)), np.ravel(st[f])), f
        assert g.time() == tm
        g.close()


@pytest.mark.parametrize("cls,transfer", [(APICMPMSolver3D, _abi.TRANSFER_APIC),
                                          (MPMSolver3D, _abi.TRANSFER_PIC_FLIP)])
def test_checkpoint_carries_cfl_and_time(gpu, tmp_path, cls, transfer):
    sc = _fast(transfer, _abi.INTERP_QUADRATIC)
    g = sc.solver()
    g.set_cfl(0.07)
    g.step(3)
    path = str(tmp_path / "cfl.ckpt")
    g.save(path)
    g.step(4)
    r = cls.from_checkpoint(path)
    r.step(4)
    for f in FIELDS:
        assert np.array_equal(g.download(f), r.download(f)), f
    # saved time + the resumed steps' sum: the same terms, grouped differently
    assert r.time()[1] == g.time()[1]
    assert r.time()[0] == pytest.approx(g.time()[0], rel=1e-12)


@pytest.mark.parametrize("bad", [np.inf, np.nan])
def test_non_finite_speed_is_reported(gpu, bad):
    """A non-finite particle velocity in a CFL scene is reported by the next
    synchronize (MPM_ERR_NUMERIC) instead of silently bounding dt by the
    finite particles (NaN) or setting it to 0 (Inf)."""
    sc = _fast(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC)
    g = sc.solver()
    g.set_cfl(0.08)
    g.step(1)
    g.synchronize()
    v = g.download(_abi.FIELD_VELOCITY)
    v[5] = bad
    g.upload(_abi.FIELD_VELOCITY, v)
    g.step(1)
    with pytest.raises(_abi.MPMError) as e:
        g.synchronize()
    assert e.value.status == 6
