"""The incremental cell-key sort (stayers kept in order, movers sorted and
merged back) returns exactly the stable sort's keys and permutation, so a run
with it (forced with MPM_INCREMENTAL_SORT=1; by default it is used from 3M
keys) is bitwise the run that sorts all keys every step (MPM_FULL_SORT=1)."""
import os

import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from mpm_b200.batch import Batch

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE, _abi.FIELD_FP)


def _run(make, steps, full_sort):
    var = "MPM_FULL_SORT" if full_sort else "MPM_INCREMENTAL_SORT"
    os.environ[var] = "1"
    try:
        eng = make()  # the engine reads the switch when it is created
    finally:
        os.environ.pop(var, None)
    eng.step(steps)
    return eng


@pytest.mark.parametrize("name", ["snow_cube", "two_balls"])
def test_incremental_sort_equals_full_sort(gpu, name):
    sc = getattr(scenes, name)()
    steps = 40 if name == "snow_cube" else 15
    a = _run(sc.solver, steps, full_sort=False)
    b = _run(sc.solver, steps, full_sort=True)
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()


def test_incremental_sort_equals_full_sort_in_a_batch(gpu):
    scs = scenes.batched_scenes(count=6, scale=0.05)

    def make():
        bt = Batch()
        bt.ids = [bt.add(s) for s in scs]
        return bt

    a = _run(make, 25, full_sort=False)
    b = _run(make, 25, full_sort=True)
    for sid_a, sid_b in zip(a.ids, b.ids):
        for f in FIELDS:
            assert np.array_equal(a.download(sid_a, f), b.download(sid_b, f)), (sid_a, f)
    a.close()
    b.close()
