"""Regenerate tests/golden/oracle_golden.json.

The reference ships no golden vectors and cannot be built here, so these
fixtures are outputs of the committed CPU oracle on small seeded scenes.  They
pin the oracle against accidental change (tests/test_oracle.py) and give the
GPU tests a fixed expectation that does not need the oracle library at run
time (tests/test_gpu_parity.py).
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mpm_b200 import _abi, scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [
    dict(name="flip_quadratic", seed=11, n=600, res=16, transfer=0, interp=1, steps=5),
    dict(name="flip_cubic", seed=12, n=600, res=16, transfer=0, interp=2, steps=5),
    dict(name="flip_linear", seed=13, n=600, res=16, transfer=0, interp=0, steps=5),
    dict(name="apic_quadratic", seed=14, n=600, res=16, transfer=1, interp=1, steps=5),
    dict(name="apic_cubic", seed=15, n=600, res=16, transfer=1, interp=2, steps=5),
]
KEEP = 64  # particles stored per field


def main():
    out = {"generator": "tests/golden/make_golden.py", "cases": []}
    for c in CASES:
        for bits in (64, 32):
            sc = scenes.tiny_scene(seed=c["seed"], n=c["n"], res=c["res"], transfer=c["transfer"],
                                   interpolation=c["interp"])
            o = O.OracleSolver(sc.desc(), sc.particles, bits=bits)
            o.step(c["steps"])
            case = dict(c, bits=bits)
            case["x"] = o.get(_abi.FIELD_POSITION).reshape(-1)[: 3 * KEEP].tolist()
            case["v"] = o.get(_abi.FIELD_VELOCITY).reshape(-1)[: 3 * KEEP].tolist()
            case["detFe"] = o.get(_abi.FIELD_DET_FE).reshape(-1)[:KEEP].tolist()
            out["cases"].append(case)
    with open(os.path.join(HERE, "oracle_golden.json"), "w") as f:
        json.dump(out, f, indent=0)


if __name__ == "__main__":
    main()
