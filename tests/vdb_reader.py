"""Reader of the OpenVDB files the library writes (test infrastructure).

Parses the OpenVDB file format (file version >= 222: per-grid compression
word, per-node metadata byte) for float grids of the standard 5-4-3 tree:
header, file and grid metadata, grid descriptors with their stream
positions, the uniform-scale transform, root tiles and children, internal
node masks and values, and leaf buffers with active-mask compression (no zip
or blosc).  It checks the structure as it goes and returns the active voxels.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = 0x56444220
COMPRESS_ZIP, COMPRESS_ACTIVE_MASK, COMPRESS_BLOSC = 1, 2, 4
NO_MASK_OR_INACTIVE_VALS, NO_MASK_AND_ALL_VALS = 0, 6


class Reader:
    def __init__(self, data: bytes):
        self.d = data
        self.p = 0

    def take(self, n):
        assert self.p + n <= len(self.d), "truncated file"
        b = self.d[self.p:self.p + n]
        self.p += n
        return b

    def u(self, fmt):
        return struct.unpack("<" + fmt, self.take(struct.calcsize("<" + fmt)))

    def string(self):
        (n,) = self.u("I")
        return self.take(n).decode()


def _mask(r, log2):
    words = np.frombuffer(r.take((1 << (3 * log2)) // 8), dtype="<u8")
    bits = np.unpackbits(words.view(np.uint8), bitorder="little").astype(bool)
    return bits  # bit i = offset i


def _values(r, count, value_mask, compression, background):
    (meta,) = r.u("b")
    if compression & COMPRESS_ACTIVE_MASK and meta != NO_MASK_AND_ALL_VALS:
        assert meta == NO_MASK_OR_INACTIVE_VALS, "only background inactive values are written"
        active = np.flatnonzero(value_mask)
        vals = np.full(count, background, np.float32)
        vals[active] = np.frombuffer(r.take(4 * active.size), dtype="<f4")
        return vals
    assert meta == NO_MASK_AND_ALL_VALS
    return np.frombuffer(r.take(4 * count), dtype="<f4").copy()


def _meta(r):
    out = {}
    (count,) = r.u("I")
    for _ in range(count):
        name, typ = r.string(), r.string()
        (size,) = r.u("I")
        raw = r.take(size)
        if typ == "string":
            out[name] = raw.decode()
        elif typ == "vec3i":
            out[name] = struct.unpack("<3i", raw)
        elif typ == "int64":
            out[name] = struct.unpack("<q", raw)[0]
        else:
            out[name] = raw
    return out


def read_vdb(path):
    """Returns a dict: header fields, grids [{name, type, meta, transform,
    background, voxels: {(x, y, z): value}, leaves}]."""
    r = Reader(open(path, "rb").read())
    (magic,) = r.u("q")
    assert magic == MAGIC, hex(magic)
    version, lib_major, lib_minor = r.u("III")
    assert version >= 222
    (offsets,) = r.u("b")
    uuid = r.take(36).decode()
    assert len(uuid.split("-")) == 5
    out = {"version": version, "library": (lib_major, lib_minor), "uuid": uuid, "meta": _meta(r), "grids": []}
    (ngrids,) = r.u("i")
    for _ in range(ngrids):
        g = {"unique_name": r.string(), "type": r.string(), "parent": r.string()}
        grid_pos, block_pos, end_pos = r.u("qqq")
        assert grid_pos == r.p, "grid position"
        (compression,) = r.u("I")
        assert not compression & (COMPRESS_ZIP | COMPRESS_BLOSC)
        g["meta"] = _meta(r)
        g["map"] = r.string()
        g["transform"] = np.frombuffer(r.take(5 * 24), dtype="<f8").reshape(5, 3)
        (nbuf,) = r.u("i")
        assert nbuf == 1
        (bg,) = r.u("f")
        ntiles, nchildren = r.u("II")
        for _ in range(ntiles):
            r.take(12 + 4 + 1)
        leaves = []  # (origin, value mask) in topology order
        for _ in range(nchildren):
            o2 = np.array(r.u("3i"))
            c2 = _mask(r, 5)
            v2 = _mask(r, 5)
            _values(r, 1 << 15, v2, compression, bg)
            for i2 in np.flatnonzero(c2):
                org1 = o2 + 128 * np.array([i2 >> 10, (i2 >> 5) & 31, i2 & 31])
                c1 = _mask(r, 4)
                v1 = _mask(r, 4)
                _values(r, 1 << 12, v1, compression, bg)
                for i1 in np.flatnonzero(c1):
                    org0 = org1 + 8 * np.array([i1 >> 8, (i1 >> 4) & 15, i1 & 15])
                    leaves.append((org0, _mask(r, 3)))
        assert block_pos == r.p, "block position"
        voxels = {}
        for org0, topo_mask in leaves:
            m = _mask(r, 3)
            assert np.array_equal(m, topo_mask)
            vals = _values(r, 512, m, compression, bg)
            for i in np.flatnonzero(m):
                voxels[(int(org0[0] + (i >> 6)), int(org0[1] + ((i >> 3) & 7)), int(org0[2] + (i & 7)))] = float(vals[i])
        assert end_pos == r.p, "end position"
        g.update(background=bg, voxels=voxels, leaves=len(leaves))
        out["grids"].append(g)
    assert r.p == len(r.d), "trailing bytes"
    return out
