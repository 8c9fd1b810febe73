"""CFL time step in the oracle: each step's dt is min(dt, cfl h / max|v_p|)
from the velocities the step starts with, and the simulated time sums them."""
import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from oracle import oracle as O


@pytest.mark.parametrize("bits", [32, 64])
def test_cfl_dt_follows_the_fastest_particle(bits):
    sc = scenes.tiny_scene(n=500, res=16, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC,
                           velocity=(0.0, -30.0, 0.0))
    o = O.OracleSolver(sc.desc(), sc.particles, bits=bits)
    o.set_cfl(0.05)
    t = 0.0
    for _ in range(4):
        v = o.get(_abi.FIELD_VELOCITY)
        want = min(sc.dt, 0.05 * sc.stride / np.sqrt((v.astype(np.float64) ** 2).sum(1).max()))
        o.step(1)
        tt, dt = o.time()
        assert dt == pytest.approx(want, rel=1e-6)
        assert dt < sc.dt
        t += dt
        assert tt == pytest.approx(t, rel=1e-12)


def test_slow_scene_keeps_the_fixed_dt():
    sc = scenes.tiny_scene(n=300, res=16, velocity=(0.0, -0.1, 0.0))
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    o.set_cfl(0.5)
    o.step(3)
    t, dt = o.time()
    assert dt == np.float64(np.float32(sc.dt))
    assert t == pytest.approx(3 * np.float64(np.float32(sc.dt)), rel=1e-12)


def test_cfl_off_is_the_plain_run():
    sc = scenes.tiny_scene(n=300, res=16, velocity=(0.0, -30.0, 0.0))
    a = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    b = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    a.set_cfl(0.0)
    a.step(3)
    b.step(3)
    assert np.array_equal(a.get(_abi.FIELD_POSITION), b.get(_abi.FIELD_POSITION))
