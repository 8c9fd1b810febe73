"""Checkpoint files are checked on the host before any device work (no GPU
needed for these cases)."""
import ctypes as C

from mpm_b200 import _abi


def _load(path):
    lib = _abi.load()
    h = C.c_void_p()
    st = lib.mpm_solver_load(str(path).encode(), C.byref(h))
    return _abi.STATUS_NAMES[st], lib.mpm_last_error_string().decode()


def test_missing_checkpoint_is_io_error(tmp_path):
    st, msg = _load(tmp_path / "nope.ckpt")
    assert st == "IO" and "cannot open" in msg


def test_garbage_checkpoint_is_parse_error(tmp_path):
    p = tmp_path / "bad.ckpt"
    p.write_bytes(b"not a checkpoint at all" * 10)
    st, msg = _load(p)
    assert st == "PARSE" and "not a checkpoint" in msg


def test_truncated_checkpoint_is_parse_error(tmp_path):
    p = tmp_path / "short.ckpt"
    p.write_bytes(b"MPMB200\x00" + (1).to_bytes(4, "little") + C.sizeof(_abi.SceneDesc).to_bytes(4, "little") + b"\x00" * 8)
    st, msg = _load(p)
    assert st == "PARSE"
