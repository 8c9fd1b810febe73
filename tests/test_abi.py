"""The C ABI library loads, exports every declared entry point, its structs
match the header layout, and argument validation works without a GPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from mpm_b200 import _abi
from mpm_b200.solver import Material, Particles, scene_desc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("mpm_b200.h", "mpm_b200_batch.h", "mpm_b200_config.h")]


def declared_symbols():
    names = []
    for h in HEADERS:
        src = open(h).read()
        names += re.findall(r"^MPM_API\s+[\w\s\*]+?\b(mpm_\w+)\s*\(", src, flags=re.M)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_symbols()
    assert len(names) >= 38
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers them all
    assert set(names) <= set(_abi.SIGNATURES)


def test_no_cuda_driver_link_dependency():
    out = subprocess.run(["ldd", _abi.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcuda.so" not in out and "libtorch" not in out


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "mpm_b200.h"\n'
        "int main(){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(mpm_material), sizeof(mpm_scene_desc),"
        " sizeof(mpm_particles_in), offsetof(mpm_scene_desc, transfer), offsetof(mpm_particles_in, materials),"
        " offsetof(mpm_scene_desc, particles_collision)); return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(_abi.Material), C.sizeof(_abi.SceneDesc), C.sizeof(_abi.ParticlesIn),
            _abi.SceneDesc.transfer.offset, _abi.ParticlesIn.materials.offset,
            _abi.SceneDesc.particles_collision.offset]
    assert got == want


def _create(desc, particles):
    lib = _abi.load()
    pin, keep = particles.to_c()
    h = C.c_void_p()
    st = lib.mpm_solver_create(C.byref(desc), C.byref(pin), C.byref(h))
    return st, lib.mpm_last_error_string().decode()


def _particles(n=8):
    x = np.random.default_rng(0).random((n, 3)).astype(np.float32) * 0.5 + 0.25
    return Particles(x, (0, 0, 0), 1.0, [Material()])


@pytest.mark.parametrize("bad", ["res", "stride", "dt", "interp", "apic_linear", "poisson", "model"])
def test_invalid_arguments_are_rejected_before_any_device_call(bad):
    d = scene_desc((0, 0, 0), (16, 16, 16), 1 / 16, 0.9, 0.95, _abi.INTERP_CUBIC, 1e-4,
                   transfer=_abi.TRANSFER_PIC_FLIP)
    p = _particles()
    if bad == "res":
        d.resolution[1] = 0
    elif bad == "stride":
        d.stride = -1.0
    elif bad == "dt":
        d.dt = float("nan")
    elif bad == "interp":
        d.interpolation = 7
    elif bad == "apic_linear":
        d.transfer = _abi.TRANSFER_APIC
        d.interpolation = _abi.INTERP_LINEAR
    elif bad == "poisson":
        p.materials[0].poisson_ratio = 0.5
    elif bad == "model":
        p.materials[0].model = 5
    st, msg = _create(d, p)
    assert st == 1, (st, msg)
    assert msg


def test_material_id_out_of_range_rejected():
    d = scene_desc((0, 0, 0), (16, 16, 16), 1 / 16, 0.9, 0.95, _abi.INTERP_QUADRATIC, 1e-4,
                   transfer=_abi.TRANSFER_PIC_FLIP)
    p = _particles()
    p.materials = [Material(), Material()]
    p.material = np.full(p.n, 2, np.uint16)
    st, msg = _create(d, p)
    assert st == 1 and "material" in msg


def test_sort_keys_rejects_bad_bits():
    lib = _abi.load()
    k = (C.c_uint32 * 4)(3, 2, 1, 0)
    o = (C.c_uint32 * 4)()
    assert lib.mpm_sort_keys(k, 4, 0, o, o) == 1
    assert lib.mpm_sort_keys(k, 4, 33, o, o) == 1


def test_solver_refuses_to_run_without_gpu_or_library():
    if _abi.device_count() > 0:
        pytest.skip("a GPU is present")
    from mpm_b200 import MPMSolver3D
    with pytest.raises(RuntimeError, match="CUDA device"):
        MPMSolver3D(_particles(), (0, 0, 0), (16, 16, 16), 1 / 16, 0.9, 0.95, 1, 1e-4)
