"""Density output (the grid the reference's writeToOpenVDB rasterises,
src/mpm_solver3d.cu:509-572): sum_p m_p w_ip / h^3 per node, checked against
the FP64 oracle's node masses; downloading it does not change the run."""
import numpy as np
import pytest

from conftest import relerr
from mpm_b200 import _abi, scenes
from mpm_b200.batch import Batch
from oracle import oracle as O

pytestmark = pytest.mark.gpu

COMBOS = [(_abi.TRANSFER_APIC, _abi.INTERP_CUBIC), (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_QUADRATIC),
          (_abi.TRANSFER_PIC_FLIP, _abi.INTERP_LINEAR)]


@pytest.mark.parametrize("transfer,interp", COMBOS)
def test_density_matches_oracle(gpu, transfer, interp):
    sc = scenes.tiny_scene(n=4000, res=24, transfer=transfer, interpolation=interp)
    g = sc.solver()
    o = O.OracleSolver(sc.desc(), sc.particles, bits=64)
    h = np.float32(sc.stride)

    def ref():
        o.reset_grid()
        o.particles_to_grid()
        return o.grid(_abi.GRID_MASS).reshape(-1) * (1.0 / float(h * h * h))

    # same positions: the node-mass tolerance of the parity tests
    assert relerr(g.density().reshape(-1), ref()) < 1e-6
    g.step(3)
    o.step(3)
    # after 3 steps the positions themselves differ within the step tolerance
    got = g.density().reshape(-1)
    assert relerr(got, ref()) < 1e-4
    # total mass is conserved by the rasterisation (partition of unity)
    total = got.astype(np.float64).sum() * float(h) ** 3
    assert abs(total / sc.particles.mass.astype(np.float64).sum() - 1) < 1e-5
    g.close()


def test_density_does_not_change_the_run(gpu):
    sc = scenes.snow_cube()
    a, b = sc.solver(), sc.solver()
    for k in range(6):
        a.step(2)
        b.step(2)
        if k % 2 == 0:
            a.density()
    for f in (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_FE):
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()


def test_batch_density_equals_solo(gpu):
    scs = scenes.batched_scenes(count=4, scale=0.05)
    with Batch() as bt:
        ids = [bt.add(s) for s in scs]
        bt.step(5)
        dens = [bt.density(i) for i in ids]
    for sc, d in zip(scs, dens):
        g = sc.solver()
        g.step(5)
        assert np.array_equal(g.density(), d)
        g.close()


def test_write_vdb_matches_density(gpu, tmp_path):
    """writeToOpenVDB (solver) and write_vdb (batch) write the density grid
    of the current state: read back, the active voxels hold exactly the
    downloaded density and every non-zero node is active."""
    from vdb_reader import read_vdb
    from mpm_b200.batch import Batch
    sc = scenes.tiny_scene(n=5000, res=24, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_CUBIC)
    g = sc.solver()
    g.step(3)
    g.writeToOpenVDB(str(tmp_path / "s.vdb"))
    rho = g.density()  # (z, y, x)
    vox = read_vdb(tmp_path / "s.vdb")["grids"][0]["voxels"]
    dense = np.zeros_like(rho)
    for (x, y, z), v in vox.items():
        dense[z, y, x] = v
    assert np.array_equal(dense, rho) and len(vox) == int(np.count_nonzero(rho))
    with Batch() as b:
        sid = b.add(sc)
        b.step(3)
        b.write_vdb(sid, str(tmp_path / "b.vdb"))
    assert read_vdb(tmp_path / "b.vdb")["grids"][0]["voxels"] == vox
