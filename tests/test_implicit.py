"""Semi-implicit update in the oracle (the reference's solveLinearSystem is a
TODO, src/mpm_solver3d.cu:312-314; the method follows Stomakhin et al. 2013,
section 9).  The Hessian action is checked against central differences of the
grid force built from the stress functions (volumeTimesCauchyStress), so the
stress differential is pinned to the same energy; the solve against its own
linear system."""
import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from mpm_b200.solver import Material
from oracle import oracle as O


def _scene(model=0, n=400, seed=3):
    sc = scenes.tiny_scene(n=n, res=16, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC)
    sc.particles.materials[0].model = model
    rng = np.random.default_rng(seed)
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    Fe = np.eye(3)[None] + 0.05 * rng.normal(size=(sc.n, 3, 3))
    Fp = np.eye(3)[None] + 0.01 * rng.normal(size=(sc.n, 3, 3))
    o.set(_abi.FIELD_FE, Fe.reshape(sc.n, 9))
    o.set(_abi.FIELD_FP, Fp.reshape(sc.n, 9))
    return sc, o


def _nodes(o):
    return o.res[0] * o.res[1] * o.res[2]


@pytest.mark.parametrize("model", [_abi.MODEL_FIXED_COROTATED, _abi.MODEL_NEO_HOOKEAN])
def test_hessian_action_is_the_force_derivative(model):
    sc, o = _scene(model)
    rng = np.random.default_rng(11)
    u = rng.normal(size=(_nodes(o), 3))
    Hu = o.hessian_action(u)
    eps = 1e-6
    fd = -(o.displaced_force(eps * u) - o.displaced_force(-eps * u)) / (2 * eps)
    assert np.abs(Hu).max() > 0
    assert np.abs(Hu - fd).max() < 1e-6 * np.abs(Hu).max()


@pytest.mark.parametrize("model", [_abi.MODEL_FIXED_COROTATED, _abi.MODEL_NEO_HOOKEAN])
def test_hessian_is_symmetric(model):
    sc, o = _scene(model)
    rng = np.random.default_rng(12)
    u, v = rng.normal(size=(2, _nodes(o), 3))
    a = (u * o.hessian_action(v)).sum()
    b = (v * o.hessian_action(u)).sum()
    assert abs(a - b) < 1e-10 * max(abs(a), 1.0)


def _grid_up_to_collision(o, dt):
    o.reset_grid()
    o.particles_to_grid()
    o.gravity()
    o.update_grid_velocities(dt)
    o.grid_collision(dt)


def test_solve_satisfies_the_system():
    sc, o = _scene()
    dt = 5e-4
    _grid_up_to_collision(o, dt)
    m = o.grid(_abi.GRID_MASS)
    vs = o.grid(_abi.GRID_VELOCITY_STAR).copy()
    o.set_implicit(1.0, max_iter=500, tol=1e-12)
    o.solve_linear_system(dt)
    it, res = o.solve_info()
    assert 0 < it < 100 and res <= 1e-12
    x = o.grid(_abi.GRID_VELOCITY_STAR)
    act = m > np.finfo(np.float32).eps
    xm = np.where(act[:, None], x, 0.0)
    r = (m[:, None] * xm + dt * dt * o.hessian_action(xm) - m[:, None] * vs)[act]
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm((m[:, None] * vs)[act])
    # the solve changed the velocities, and left massless nodes alone
    assert np.abs(x[act] - vs[act]).max() > 1e-3 * np.abs(vs[act]).max()
    assert np.array_equal(x[~act], vs[~act])


def test_beta_zero_is_explicit():
    sc, o = _scene()
    _, p = _scene()
    o.set_implicit(0.0)
    o.step(3)
    p.step(3)
    assert np.array_equal(o.get(_abi.FIELD_POSITION), p.get(_abi.FIELD_POSITION))
    dt = sc.dt
    _grid_up_to_collision(o, dt)
    before = o.grid(_abi.GRID_VELOCITY_STAR).copy()
    o.solve_linear_system(dt)
    assert np.array_equal(o.grid(_abi.GRID_VELOCITY_STAR), before)


def jelly(dt=1e-3, n=500):
    """A stiff elastic block (E = 1e6, plasticity limits far away) with random
    velocities, at 5x the explicit stability limit of its 16^3 grid."""
    sc = scenes.tiny_scene(n=n, res=16, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_QUADRATIC,
                           gravity=0.0, velocity=(0.0, 0.0, 0.0))
    m = sc.particles.materials[0]
    m.youngs_modulus, m.critical_compression, m.critical_stretch, m.hardening = 1e6, 0.9, 4.0, 0.0
    sc.particles.velocities = (0.5 * np.random.default_rng(1).normal(size=(sc.n, 3))).astype(np.float32)
    sc.dt = dt
    return sc


def test_implicit_is_stable_where_explicit_blows_up():
    sc = jelly()
    vmax = {}
    for beta in (0.0, 1.0):
        o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
        o.set_implicit(beta, max_iter=100, tol=1e-8)
        o.step(40)
        v = o.get(_abi.FIELD_VELOCITY)
        vmax[beta] = np.abs(v).max() if np.isfinite(v).all() else np.inf
    assert vmax[0.0] > 100.0
    assert vmax[1.0] < 0.5


@pytest.mark.parametrize("model", [_abi.MODEL_FIXED_COROTATED, _abi.MODEL_NEO_HOOKEAN])
def test_hessian_at_large_strain(model):
    """20 % deformations (rotation differential far from the identity)."""
    sc = scenes.tiny_scene(n=300, res=16, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_CUBIC)
    sc.particles.materials[0].model = model
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    rng = np.random.default_rng(21)
    A = rng.normal(size=(sc.n, 3, 3))
    Q, _ = np.linalg.qr(A)
    Q *= np.sign(np.linalg.det(Q))[:, None, None]  # proper rotations
    Fe = Q @ (np.eye(3)[None] + 0.2 * rng.normal(size=(sc.n, 3, 3)))
    o.set(_abi.FIELD_FE, Fe.reshape(sc.n, 9))
    u = rng.normal(size=(_nodes(o), 3))
    Hu = o.hessian_action(u)
    eps = 1e-6
    fd = -(o.displaced_force(eps * u) - o.displaced_force(-eps * u)) / (2 * eps)
    assert np.abs(Hu - fd).max() < 1e-6 * np.abs(Hu).max()


def test_hessian_rows_sum_to_zero_and_solve_conserves_momentum():
    """The elastic energy is translation-invariant: sum_i (H u)_i = 0 for any
    u over all nodes.  The solve's unknowns are the nodes with m > FLT_EPSILON
    (the velocity update's threshold); the few lighter nodes at the edge of the
    stencils drop their share of H x, so the grid momentum sum_i m_i v_i is
    kept to ~1e-6 relative, not exactly."""
    sc, o = _scene(seed=8)
    rng = np.random.default_rng(4)
    u = rng.normal(size=(_nodes(o), 3))
    Hu = o.hessian_action(u)
    assert np.abs(Hu.sum(0)).max() < 1e-9 * np.abs(Hu).max()
    dt = 1e-3
    o.reset_grid()
    o.particles_to_grid()
    o.update_grid_velocities(dt)  # no gravity, no boundary: only the elastic forces act
    m = o.grid(_abi.GRID_MASS)
    act = m > np.finfo(np.float32).eps
    vs = o.grid(_abi.GRID_VELOCITY_STAR).copy()
    o.set_implicit(1.0, max_iter=500, tol=1e-13)
    o.solve_linear_system(dt)
    v = o.grid(_abi.GRID_VELOCITY_STAR)
    p0 = (m[act, None] * vs[act]).sum(0)
    p1 = (m[act, None] * v[act]).sum(0)
    assert np.abs(p1 - p0).max() < 1e-5 * np.abs(p0).max()
    assert np.abs(v[act] - vs[act]).max() > 1e-3 * np.abs(vs[act]).max()  # the solve acted
