"""OpenVDB output of the density grid (no GPU needed): the library's writer
(mpm_write_vdb_density) read back by tests/vdb_reader.py.  The density is the
oracle's node mass / h^3 after its P2G -- the grid the reference's
writeToOpenVDB rasterises (src/mpm_solver3d.cu:509-572)."""
import ctypes as C

import numpy as np
import pytest

from mpm_b200 import _abi, scenes
from oracle import oracle as O
from vdb_reader import read_vdb


def _write(density, res, path):
    lib = _abi.load()
    d = np.ascontiguousarray(density, np.float32).reshape(-1)
    r = (C.c_int32 * 3)(*res)
    _abi.check(lib.mpm_write_vdb_density(d.ctypes.data_as(C.POINTER(C.c_float)), r, str(path).encode()),
               "mpm_write_vdb_density")


def _dense(vox, res):
    out = np.zeros(res[::-1], np.float32)  # (z, y, x)
    for (x, y, z), v in vox.items():
        out[z, y, x] = v
    return out


def test_oracle_density_round_trip(tmp_path):
    sc = scenes.tiny_scene(n=3000, res=24, transfer=_abi.TRANSFER_APIC, interpolation=_abi.INTERP_CUBIC)
    o = O.OracleSolver(sc.desc(), sc.particles, bits=32)
    o.reset_grid()
    o.particles_to_grid()
    rho = (o.grid(_abi.GRID_MASS) / sc.stride ** 3).astype(np.float32)
    res = sc.resolution
    _write(rho, res, tmp_path / "d.vdb")
    f = read_vdb(tmp_path / "d.vdb")
    assert f["version"] == 224 and len(f["grids"]) == 1
    g = f["grids"][0]
    assert g["unique_name"] == "density" and g["type"] == "Tree_float_5_4_3" and g["meta"]["name"] == "density"
    assert g["map"] == "UniformScaleMap" and np.array_equal(g["transform"][1], [1, 1, 1])
    assert g["background"] == 0.0
    dense = _dense(g["voxels"], res)
    assert np.array_equal(dense.reshape(-1), rho)  # bitwise
    nz = np.argwhere(rho.reshape(res[::-1]) != 0)
    assert g["meta"]["file_voxel_count"] == len(nz) == len(g["voxels"])
    assert tuple(g["meta"]["file_bbox_min"]) == tuple(nz.min(0)[::-1])
    assert tuple(g["meta"]["file_bbox_max"]) == tuple(nz.max(0)[::-1])


@pytest.mark.parametrize("res", [(8, 8, 8), (200, 9, 130), (300, 4, 5)])
def test_sparse_leaves_across_internal_nodes(tmp_path, res):
    """Voxels spread over several 8^3 leaves and 128^3 internal nodes
    (x up to 299 spans three), values of every sign, one fully active leaf."""
    rng = np.random.default_rng(sum(res))
    rho = np.zeros(res[::-1], np.float32)
    idx = rng.integers(0, rho.size, rho.size // 7)
    rho.reshape(-1)[idx] = rng.normal(size=idx.size).astype(np.float32)
    rho[:min(8, res[2]), :min(8, res[1]), :8] = 1.5
    _write(rho, res, tmp_path / "s.vdb")
    g = read_vdb(tmp_path / "s.vdb")["grids"][0]
    assert np.array_equal(_dense(g["voxels"], res), rho)


def test_empty_grid(tmp_path):
    _write(np.zeros(64, np.float32), (4, 4, 4), tmp_path / "e.vdb")
    g = read_vdb(tmp_path / "e.vdb")["grids"][0]
    assert g["voxels"] == {} and g["leaves"] == 0


def test_bad_path_reports_io_error(tmp_path):
    with pytest.raises(_abi.MPMError) as e:
        _write(np.ones(8, np.float32), (2, 2, 2), tmp_path / "no_such_dir" / "x.vdb")
    assert e.value.status == 2
