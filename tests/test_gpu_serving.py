"""Serving: continuous batching gives every request the result it gets alone."""
import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from mpm_b200.serving import Server, scene_device_bytes

pytestmark = pytest.mark.gpu


def test_each_request_matches_its_solo_run(gpu):
    reqs = scenes.serving_requests(seed=5, rate=200.0, duration=0.2, n_min=500, n_max=20_000, max_requests=10)
    for r in reqs:  # keep the check quick
        r.scene.steps = 5 + r.rid % 7
    assert len(reqs) >= 5
    srv = Server(budget_bytes=2e9)
    rep = srv.run(reqs, time_scale=1.0)
    srv.close()
    assert len(rep.results) == len(reqs) and not rep.rejected
    assert max(rep.batch_sizes) >= 2  # requests overlapped on the device
    by_id = {r.rid: r for r in rep.results}
    for req in reqs:
        g = req.scene.solver()
        g.step(req.scene.steps)
        for f, got in by_id[req.rid].state.items():
            assert np.array_equal(got, g.download(f)), (req.rid, f)
    s = rep.summary()
    assert s["p99_step_ms"] >= s["p50_step_ms"] > 0


def test_budget_admission_defers_and_rejects(gpu):
    reqs = scenes.serving_requests(seed=6, rate=500.0, duration=0.05, n_min=2000, n_max=4000, max_requests=6)
    for r in reqs:
        r.scene.steps = 3
    need = max(scene_device_bytes(r.scene) for r in reqs)
    # room for one scene at a time: requests queue, run one after another
    srv = Server(budget_bytes=need * 1.01)
    rep = srv.run(reqs)
    srv.close()
    assert len(rep.results) == len(reqs)
    assert max(rep.batch_sizes) < len(reqs)  # some requests waited for memory
    # a budget below every scene rejects all requests instead of hanging
    srv = Server(budget_bytes=1.0)
    rep = srv.run(reqs)
    srv.close()
    assert len(rep.rejected) == len(reqs) and not rep.results


def test_release_cached_memory_between_solvers(gpu):
    """Scene memory comes from a pool that keeps freed blocks; releasing the
    cache between solvers leaves later solvers working and bitwise equal."""
    lib = _abi.load()
    sc = scenes.tiny_scene(n=2048, res=16)
    g = sc.solver()
    g.step(3)
    x0 = g.download(_abi.FIELD_POSITION)
    g.close()
    _abi.check(lib.mpm_release_cached_memory(0), "mpm_release_cached_memory")
    g = sc.solver()
    g.step(3)
    assert np.array_equal(g.download(_abi.FIELD_POSITION), x0)
    g.close()
    assert _abi.STATUS_NAMES[lib.mpm_release_cached_memory(-1)] == "INVALID_ARG"
