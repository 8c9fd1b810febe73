"""The optional step features together: a level-set obstacle, the CFL time
step and the semi-implicit update in one run, against the FP64 oracle doing
the same, and a batch of such scenes against their solo runs."""
import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, level_set, scenes
from mpm_b200.batch import Batch
from mpm_b200.level_set import LevelSetCollisionObject3D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP)


def _scene(seed=7, v=(0.5, -20.0, 0.25)):
    sc = scenes.tiny_scene(seed=seed, n=4000, res=24, transfer=_abi.TRANSFER_APIC,
                           interpolation=_abi.INTERP_QUADRATIC, velocity=v)
    sc.dt = 5e-4  # the CFL limit below is the smaller one
    phi = level_set.sphere(sc.origin, sc.resolution, sc.stride, (0.45, 0.2, 0.45), 0.12)
    return sc, LevelSetCollisionObject3D(phi, friction=0.4, velocity=(0.1, 0.0, 0.0))


def test_level_set_cfl_implicit_match_oracle(gpu):
    sc, obj = _scene()
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    g.set_collision_object(obj)
    o.set_level_set(obj.level_set, obj.friction, obj.velocity)
    g.set_cfl(0.2)
    o.set_cfl(0.2)
    g.set_implicit(1.0, max_iter=200, tol=1e-6)
    o.set_implicit(1.0, max_iter=500, tol=1e-12)
    g.step(4)
    o.step(4)
    tg, dg = g.time()
    to, do = o.time()
    assert dg < sc.dt and abs(dg / do - 1) < 1e-4 and abs(tg / to - 1) < 1e-4
    it, res = g.solve_info()
    assert it > 0 and res <= 1e-6
    for f in FIELDS:
        assert relerr(g.download(f), o.get(f)) < 1e-4, f


def test_batch_with_all_features_equals_solo(gpu):
    built = [_scene(seed=s, v=(0.3 * s, -15.0 - s, 0.1)) for s in (3, 4, 5)]
    with Batch() as bt:
        ids = [bt.add(sc) for sc, _ in built]
        for sid, (sc, obj) in zip(ids, built):
            bt.set_collision_object(sid, obj)
            bt.set_cfl(sid, 0.2)
            bt.set_implicit(sid, 1.0, max_iter=40, tol=1e-6)
        bt.step(6)
        got = [([bt.download(sid, f) for f in FIELDS], bt.time(sid), bt.solve_info(sid)) for sid in ids]
    for (sc, obj), (st, tm, inf) in zip(built, got):
        g = sc.solver()
        g.set_collision_object(obj)
        g.set_cfl(0.2)
        g.set_implicit(1.0, max_iter=40, tol=1e-6)
        g.step(6)
        for f, x in zip(FIELDS, st):
            assert np.array_equal(np.ravel(g.download(f)), np.ravel(x)), f
        assert g.time() == tm and g.solve_info() == inf
        g.close()
