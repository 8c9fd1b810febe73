"""Copy the reference's own scene fixtures into tests/golden/reference/.

The reference ships five YAML scene configurations (config/*.yaml) and three
sparse point clouds (data/*_sparse.xyz).  The tests parse all five YAMLs with
the library's reader and run the snow-cube scene (config/snow_cube.yaml with
data/cube_sparse.xyz: 11,907 points on integer grid coordinates, 200^3 grid,
cubic B-spline, PIC-FLIP) on the GPU against the oracle.  The tests read the
copies here, so nothing at test time depends on a checkout of the reference.
The two-ball point clouds (data/ball1_sparse.xyz, data/ball2_sparse.xyz: 6,101
and 56,907 points, 2.7 MB of text) are stored gzip-compressed as *.xyz.gz
(196 KB); the tests that run config/snow_two_balls_sparse.yaml unpack them
next to a copy of the YAML.

Run from the repository root with the reference checkout as the argument:
    python tests/golden/reference/vendor.py <reference checkout>
The copies are byte-for-byte; the directory layout (config/ beside data/)
keeps the YAMLs' relative `File: ../data/...` paths valid.
"""
import gzip
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CONFIGS = ["snow_cube.yaml", "snow_two_balls_sparse.yaml", "snow_two_balls.yaml", "snow_text.yaml",
           "snow_cylinder_dragon.yaml"]
DATA = ["cube_sparse.xyz"]
DATA_GZ = ["ball1_sparse.xyz", "ball2_sparse.xyz"]


def main(ref_root: str) -> None:
    for sub, names in (("config", CONFIGS), ("data", DATA)):
        os.makedirs(os.path.join(HERE, sub), exist_ok=True)
        for name in names:
            shutil.copyfile(os.path.join(ref_root, sub, name), os.path.join(HERE, sub, name))
            print("copied", os.path.join(sub, name))
    for name in DATA_GZ:
        with open(os.path.join(ref_root, "data", name), "rb") as f:
            raw = f.read()
        with open(os.path.join(HERE, "data", name + ".gz"), "wb") as f:
            f.write(gzip.compress(raw, compresslevel=9, mtime=0))
        print("copied", os.path.join("data", name + ".gz"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
