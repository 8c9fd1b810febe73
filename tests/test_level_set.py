"""Level-set collision objects on the CPU: known answers of the oracle's
collision rule (the friction law of applyBoundaryCollision,
src/collision_object3d.cu:38-51, on a level set), the signed-distance builders,
and an oracle run of a ball falling onto a sphere obstacle."""
import numpy as np
import pytest

from mpm_b200 import _abi, level_set, scenes
from oracle import oracle as O

RES = (8, 8, 8)
H = 1.0 / 8
ORIGIN = (0.0, 0.0, 0.0)


def _plane_y(y0):
    return level_set.half_space(ORIGIN, RES, H, (0.0, y0, 0.0), (0.0, 1.0, 0.0))


def _friction_law(v, n, mu, vco=(0.0, 0.0, 0.0)):
    rel = np.asarray(v, float) - vco
    vn = rel @ n
    if vn >= np.finfo(np.float32).eps:
        return np.asarray(v, float)
    vt = rel - vn * n
    if np.linalg.norm(vt) <= -mu * vn + np.finfo(np.float32).eps:
        return np.asarray(vco, float)
    return vt + mu * vn * vt / np.linalg.norm(vt) + vco


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("v,mu,vco", [((1.0, -2.0, 0.5), 0.3, (0, 0, 0)), ((0.1, -2.0, 0.0), 1.0, (0, 0, 0)),
                                      ((0.8, -3.0, 0.2), 0.2, (0.5, 0.0, -0.1)), ((0.0, 1.0, 0.0), 0.5, (0, 0, 0))])
def test_plane_known_answers(bits, v, mu, vco):
    phi = _plane_y(0.5)
    got = O.level_set_collision(bits, RES, ORIGIN, H, phi, mu, vco, (0.31, 0.45, 0.62), v)
    want = _friction_law(v, np.array([0.0, 1.0, 0.0]), mu, np.asarray(vco, float))
    assert np.allclose(got, want, rtol=0, atol=1e-6 if bits == 32 else 1e-12)


def test_outside_is_untouched():
    phi = _plane_y(0.5)
    v = (1.0, -2.0, 0.5)
    got = O.level_set_collision(64, RES, ORIGIN, H, phi, 0.4, (0, 0, 0), (0.3, 0.55, 0.3), v)
    assert np.array_equal(got, np.asarray(v))


def test_positions_outside_the_grid_are_clamped():
    phi = _plane_y(0.5)
    # below the grid: clamped to the y = 0 layer (inside), normal +y
    got = O.level_set_collision(64, RES, ORIGIN, H, phi, 0.0, (0, 0, 0), (-0.5, -1.0, 2.0), (0.3, -1.0, 0.0))
    assert np.allclose(got, (0.3, 0.0, 0.0), atol=1e-12)


def test_oblique_plane_normal():
    n = np.array([1.0, 2.0, -0.5])
    n /= np.linalg.norm(n)
    phi = level_set.half_space(ORIGIN, RES, H, (0.5, 0.5, 0.5), n)
    v = (-1.0, -0.5, 0.7)
    got = O.level_set_collision(64, RES, ORIGIN, H, phi, 0.25, (0, 0, 0), (0.4, 0.45, 0.5), v)
    # a linear field is reproduced exactly by trilinear interpolation, and so is its gradient
    assert np.allclose(got, _friction_law(v, n, 0.25), atol=1e-6)


def test_builders():
    res = (16, 12, 10)
    h = 0.1
    s = level_set.sphere((0, 0, 0), res, h, (0.8, 0.6, 0.5), 0.3)
    assert s.shape == (10, 12, 16) and s.dtype == np.float32
    assert s[5, 6, 8] == pytest.approx(-0.3)           # node (0.8, 0.6, 0.5)
    assert s[5, 6, 12] == pytest.approx(0.1, abs=1e-6)  # x = 1.2
    b = level_set.box((0, 0, 0), res, h, (0.2, 0.2, 0.2), (0.6, 0.6, 0.6))
    assert b[4, 4, 4] == pytest.approx(-0.2, abs=1e-6)  # centre
    assert b[2, 2, 9] == pytest.approx(0.3, abs=1e-6)   # (0.9, 0.2, 0.2): 0.3 from the x face
    assert b[0, 0, 0] == pytest.approx(np.sqrt(3) * 0.2, abs=1e-6)
    u = level_set.union(s, b)
    assert np.array_equal(u, np.minimum(s, b))
    obj = level_set.LevelSetCollisionObject3D(s, friction=0.2)
    phi, vel = obj.arrays(res)
    assert phi.size == 16 * 12 * 10 and np.array_equal(vel, np.zeros(3, np.float32))
    with pytest.raises(ValueError):
        obj.arrays((16, 12, 11))


def _falling_ball():
    sc = scenes.tiny_scene(n=600, res=16, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC,
                           velocity=(0.0, -15.0, 0.0))
    sc.dt = 2e-4
    phi = level_set.sphere(sc.origin, sc.resolution, sc.stride, (0.45, 0.12, 0.45), 0.12)
    return sc, phi


def _sample(phi, res, h, x):
    from scipy.ndimage import map_coordinates
    coords = np.stack([x[:, 2] / h, x[:, 1] / h, x[:, 0] / h])
    return map_coordinates(phi.astype(np.float64), coords, order=1, mode="nearest")


def test_oracle_ball_stays_out_of_the_obstacle():
    sc, phi = _falling_ball()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    o.set_level_set(phi, friction=0.5)
    free = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    for _ in range(6):
        o.step(10)
        free.step(10)
    x = o.get(_abi.FIELD_POSITION)
    xf = free.get(_abi.FIELD_POSITION)
    # without the obstacle the ball falls through its place
    assert _sample(phi, sc.resolution, sc.stride, xf).min() < -0.05
    # with it, no particle is more than a cell inside
    assert _sample(phi, sc.resolution, sc.stride, x).min() > -sc.stride


def test_far_obstacle_changes_nothing():
    sc, _ = _falling_ball()
    far = level_set.sphere(sc.origin, sc.resolution, sc.stride, (5.0, 5.0, 5.0), 0.1)
    a = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    b = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    a.set_level_set(far, friction=0.5)
    a.step(5)
    b.step(5)
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE):
        assert np.array_equal(a.get(f), b.get(f))
