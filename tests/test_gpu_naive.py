"""The reference-naive GPU baseline (baseline/naive) computes the same step:
checked against the FP64 oracle so that the speed-up bench.py reports is
against a correct implementation."""
import os
import sys

import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "naive"))
import naive as NV  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("transfer,interp", [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC),
                                             (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_LINEAR)])
def test_naive_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=3000, res=16, transfer=transfer, interpolation=interp)
    g = NV.NaiveSolver(sc.desc(), sc.particles)
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    assert relerr(g.download(_abi.FIELD_VOLUME0), o.get(_abi.FIELD_VOLUME0)) < 3e-6
    g.step(2)
    o.step(2)
    for f, tol in ((_abi.FIELD_POSITION, 1e-5), (_abi.FIELD_VELOCITY, 1e-4), (_abi.FIELD_FE, 1e-5),
                   (_abi.FIELD_FP, 1e-5)):
        ref = o.get(f)
        assert relerr(g.download(f).reshape(ref.shape), ref) < tol, f
    g.close()


def test_naive_two_ball_runs(gpu):
    """The benchmark scene steps on the naive baseline and stays finite."""
    sc = scenes.two_balls()
    g = NV.NaiveSolver(sc.desc(), sc.particles)
    ms = g.timed_step(3)
    x = g.download(_abi.FIELD_POSITION)
    assert ms > 0 and np.isfinite(x).all()
    g.close()
