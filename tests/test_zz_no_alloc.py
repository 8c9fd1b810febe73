"""The allocation-free sort entry point against the allocating one.

mpm_sort_keys_device_noalloc serves callers that own all device memory and do
not let the library allocate (their own pool, a fixed start-up budget, or a
loop that must not risk the implicit synchronization of cudaMalloc/cudaFree):
they pass device input and output buffers and the sort works in a fixed
device array inside the library.  The test calls it through the C ABI twice
in a row on different keys, compares each result bit for bit with
mpm_sort_keys (the allocating entry point, host buffers), and checks that an
input larger than the fixed capacity is refused.  The file name makes pytest
collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from mpm_b200 import _abi

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20  # MPM_SORT_NOALLOC_MAX_KEYS


def _reference_sort(keys, bits):
    lib = _abi.load()
    n = keys.size
    sk = np.empty(n, np.uint32)
    pm = np.empty(n, np.uint32)
    P = C.POINTER(C.c_uint32)
    _abi.check(lib.mpm_sort_keys(keys.ctypes.data_as(P), n, bits, sk.ctypes.data_as(P), pm.ctypes.data_as(P)),
               "mpm_sort_keys")
    return sk, pm


def _noalloc_sort(keys, bits):
    import torch
    lib = _abi.load()
    _abi.check(lib.mpm_set_device(0), "mpm_set_device")
    torch.cuda.set_device(0)
    n = keys.size
    d_in = torch.from_numpy(keys.view(np.int32)).cuda()
    d_keys = torch.empty(n, dtype=torch.int32, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.mpm_sort_keys_device_noalloc(C.c_void_p(d_in.data_ptr()), n, bits, C.c_void_p(d_keys.data_ptr()),
                                          C.c_void_p(d_perm.data_ptr()), C.c_void_p(stream.cuda_stream))
    _abi.check(st, "mpm_sort_keys_device_noalloc")
    stream.synchronize()
    return d_keys.cpu().numpy().view(np.uint32), d_perm.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(gpu):
    rng = np.random.default_rng(2024)
    cases = [
        (rng.integers(0, 1 << 22, MAX_KEYS, dtype=np.uint64).astype(np.uint32), 22),   # full capacity, 3 passes
        (rng.integers(0, 64, 300_001, dtype=np.uint64).astype(np.uint32) * 4099, 18),  # duplicates, 3 passes
    ]
    for keys, bits in cases:  # two calls in a row through the shared scratch
        got_k, got_p = _noalloc_sort(keys, bits)
        ref_k, ref_p = _reference_sort(keys, bits)
        assert np.array_equal(got_k, ref_k)
        assert np.array_equal(got_p, ref_p)
        assert np.array_equal(got_p, np.argsort(keys, kind="stable").astype(np.uint32))


def test_noalloc_sort_even_pass_count(gpu):
    keys = np.random.default_rng(5).integers(0, 1 << 16, 70_000, dtype=np.uint64).astype(np.uint32)
    got_k, got_p = _noalloc_sort(keys, 16)
    ref_k, ref_p = _reference_sort(keys, 16)
    assert np.array_equal(got_k, ref_k) and np.array_equal(got_p, ref_p)


def test_noalloc_sort_rejects_oversized_input(gpu):
    lib = _abi.load()
    st = lib.mpm_sort_keys_device_noalloc(C.c_void_p(1), MAX_KEYS + 1, 22, C.c_void_p(1), C.c_void_p(1), None)
    assert st == 1
    assert b"MPM_SORT_NOALLOC_MAX_KEYS" in lib.mpm_last_error_string()


@pytest.mark.parametrize("n,bits", [(1000, 8), (2049, 32), (1, 5), (2047, 12)])
def test_noalloc_sort_single_pass_and_ragged_sizes(gpu, n, bits):
    """One pass (bits <= 8: the first pass writes straight into the caller's
    outputs), inputs below one 2048-key tile, one key past a tile, and n = 1,
    each against the allocating sort and a CPU stable sort."""
    hi = (1 << bits) if bits < 32 else (1 << 32)
    keys = np.random.default_rng(n * 7 + bits).integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    got_k, got_p = _noalloc_sort(keys, bits)
    ref_k, ref_p = _reference_sort(keys, bits)
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    assert np.array_equal(got_p, ref_p) and np.array_equal(got_p, order)
    assert np.array_equal(got_k, ref_k) and np.array_equal(got_k, keys[order])


def test_noalloc_sort_rejects_overlapping_buffers(gpu):
    """An in-place call (keys == sorted_keys) or outputs that overlap are
    refused before any device work: the passes read the input while they
    scatter into the outputs."""
    lib = _abi.load()
    base = 1 << 20  # never dereferenced: the argument check comes first
    for keys, out, perm in ((base, base, base + 65536), (base, base + 4 * 999, base + 65536),
                            (base, base + 65536, base + 65536 + 4 * 100)):
        st = lib.mpm_sort_keys_device_noalloc(C.c_void_p(keys), 1000, 16, C.c_void_p(out), C.c_void_p(perm), None)
        assert st == 1
        assert b"must not overlap" in lib.mpm_last_error_string()
