"""Committed fixtures (tests/golden/tiny_substep.json, written by
tests/golden/make_golden.py from the oracle): the oracle must keep
reproducing them (CPU), and the CUDA path must reproduce them through the
C ABI without any CPU solve (GPU)."""
import json
import os
import sys

import numpy as np
import pytest

from opentbl_b200 import native, synth
from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402

with open(os.path.join(GOLDEN, "tiny_substep.json")) as f:
    FIX = json.load(f)


def _check(box, ref, rtol_l2, rtol_pt):
    um, st = box.inflow()
    for n, fp in ref["fields"].items():
        a = np.asarray(box.field(n)).ravel()
        rms = fp["l2"] / np.sqrt(a.size)
        assert abs(np.linalg.norm(a) - fp["l2"]) <= rtol_l2 * max(fp["l2"], 1e-300), n
        d = np.abs(a[fp["idx"]] - np.asarray(fp["val"]))
        assert d.max() <= rtol_pt * max(rms, 1e-300), (n, d.max(), rms)
    ua = np.asarray(um)
    assert np.abs(ua[ref["um"]["idx"]] - np.asarray(ref["um"]["val"])).max() <= rtol_pt
    for k, v in ref["scalars"].items():
        assert abs(st[k] - v) <= max(rtol_l2, 1e-14) * max(1.0, abs(v)), (k, st[k], v)


def _inputs(tag):
    cfg = make_golden.cases()[tag]
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    return cfg, init, coef


@pytest.mark.parametrize("tag", ["fp64", "real4"])
def test_oracle_reproduces_fixtures(tag):
    cfg, init, coef = _inputs(tag)
    ob = pyoracle.OracleBox(cfg, init, threads=1)
    ob.substep(1, 1)
    _check(ob, FIX[tag]["substep1"], 1e-13, 1e-12)
    ob = pyoracle.OracleBox(cfg, init, threads=1)
    ob.advance(1)
    _check(ob, FIX[tag]["step1"], 1e-13, 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["fp64", "real4"])
def test_cuda_path_reproduces_fixtures(tag):
    """FP64: 1e-11 on norms and points after one substep and one step. The
    REAL4 mode flips an occasional FP32 rounding against the oracle, so its
    bound is the single-precision one, 1e-6."""
    from opentbl_b200 import Box
    cfg, init, coef = _inputs(tag)
    tol = 1e-11 if tag == "fp64" else 1e-6
    g = Box(cfg, init, coef)
    g.substep(1, True)
    _check(g, FIX[tag]["substep1"], tol, 10 * tol)
    g = Box(cfg, init, coef)
    g.advance(1)
    _check(g, FIX[tag]["step1"], tol, 10 * tol)
