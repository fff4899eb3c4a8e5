"""Writes tests/golden/tiny_substep.json: fingerprints of the oracle's state
on the seeded 33x41x32 box after one RK3 substep (m = 1, new dt) and after
one full RK3 step, in FP64 and in REAL4-transpose mode.

The reference ships no test data and its Fortran cannot be built here, so
these fixtures come from the oracle (oracle/); they pin the oracle against
regressions and give the GPU tests a check that needs no CPU solve. Each
field is fingerprinted by its L2 norm, its plain sum and 64 values at
seeded flat indices.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from opentbl_b200 import config, synth  # noqa: E402
from opentbl_b200.config import replace  # noqa: E402
from oracle import pyoracle  # noqa: E402

FIELDS = ("u", "v", "w", "p", "rhsupa", "rhsvpa", "rhswpa")
SCALARS = ("dt", "tiempo", "utauout", "rthout", "dout", "gamma1", "gamma2", "timec")
OUT = os.path.join(HERE, "tiny_substep.json")


def sample_index(shape, n=64, seed=2024):
    rng = np.random.default_rng(seed)
    return rng.integers(0, int(np.prod(shape)), size=n).tolist()


def fingerprint(arr):
    a = np.asarray(arr, dtype=np.float64)
    idx = sample_index(a.shape)
    flat = a.ravel()
    return {"l2": float(np.linalg.norm(flat)), "sum": float(flat.sum()),
            "idx": idx, "val": [float(flat[i]) for i in idx]}


def state_fp(box):
    um, st = box.inflow()
    return {"fields": {n: fingerprint(box.field(n)) for n in FIELDS},
            "um": fingerprint(um), "scalars": {k: float(st[k]) for k in SCALARS}}


def cases():
    return {"fp64": config.TINY, "real4": replace(config.TINY, xpose_round=1)}


def make():
    out = {}
    for tag, cfg in cases().items():
        init = synth.make_initial(cfg)
        ob = pyoracle.OracleBox(cfg, init, threads=1)
        ob.substep(1, 1)
        one = state_fp(ob)
        ob.close()
        ob = pyoracle.OracleBox(cfg, init, threads=1)
        ob.advance(1)
        step = state_fp(ob)
        ob.close()
        out[tag] = {"config": cfg.name, "xpose_round": cfg.xpose_round,
                    "substep1": one, "step1": step}
    return out


if __name__ == "__main__":
    with open(OUT, "w") as f:
        json.dump(make(), f, separators=(",", ":"))
    print("wrote", OUT)
