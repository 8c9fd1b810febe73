"""The reference's two-ball scene (config/snow_two_balls_sparse.yaml with its
point clouds, vendored gzip-compressed by tests/golden/reference/vendor.py)
unpacked into a directory with the config/ + data/ layout its relative
`File: ../data/...` paths expect.  Test infrastructure."""
import gzip
import os
import shutil

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference")


def unpack_two_balls(dst: str) -> str:
    """Returns the path of the unpacked YAML under dst."""
    os.makedirs(os.path.join(dst, "config"), exist_ok=True)
    os.makedirs(os.path.join(dst, "data"), exist_ok=True)
    yml = os.path.join(dst, "config", "snow_two_balls_sparse.yaml")
    shutil.copyfile(os.path.join(REF_DIR, "config", "snow_two_balls_sparse.yaml"), yml)
    for name in ("ball1_sparse.xyz", "ball2_sparse.xyz"):
        with gzip.open(os.path.join(REF_DIR, "data", name + ".gz"), "rb") as f:
            raw = f.read()
        with open(os.path.join(dst, "data", name), "wb") as f:
            f.write(raw)
    return yml
