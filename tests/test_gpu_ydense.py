"""interpyy (lip.f90:359-440) of the mixed-precision path as a dense operator
on the tcgen05 tensor cores (OTBL_OPT_YDENSE, csrc/k_ydense.cu) against the
FP64 oracle and against the banded FP32 solve of the same path.

The dense operator Mop = A^-1 B is applied with three TF32 products
(hi*hi + hi*lo + lo*hi of the split operator and field) accumulated in FP32,
so its interpolants carry FP32-level errors like the banded FP32 sweep's.
Tolerances (written here): interpolants within 2e-6 of the oracle's FP64
interpyy relative to the field's largest value (measured FP32 banded error
about 1e-7); after one substep the velocity within 1e-6 of the oracle and
within 1e-6 of the banded mixed path; after 20 steps of 257x97x128 within
1e-6 of the oracle (the mixed path's regression bound), max|div u| <= 1e-10.
"""
import ctypes

import numpy as np
import pytest

from opentbl_b200 import Box, config
from opentbl_b200.config import replace

from helpers import oracle_box, setup
from test_gpu_mixed import _report

pytestmark = pytest.mark.gpu

D = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731


def _dense(cfg):
    return replace(cfg, precision=1, options=1, name=(cfg.name or "box") + "-mixed-ydense")


def _oracle_interpyy(cfg, o, fld, which):
    """orc_interpyy plane by plane on the oracle's own copy of the field."""
    rows_in = cfg.ny + 1 if which == 0 else cfg.ny
    out = np.zeros((cfg.nx, cfg.ny, cfg.nz1))
    for i in range(cfg.nx):
        g = np.ascontiguousarray(fld[i, :rows_in, :])
        r = np.zeros((cfg.ny + 1, cfg.nz1))
        o.L.orc_interpyy(o.h, D(g), D(r), which, cfg.nz1, cfg.nz1)
        out[i] = r[:cfg.ny]
    return out


@pytest.mark.parametrize("name", ["TINY", "SMALL", "C1", "SLAB"])
def test_ydense_interpolants_against_oracle(name):
    """TINY, C1: one tile per plane (32 and 96 columns); SMALL: nz1 = 42,
    not a multiple of 4; SLAB (257x193x512): two tiles of 176 columns per
    plane, the second partly past nz1 = 340, and two M-tiles (ny = 193)."""
    cfg = getattr(config, name)
    init, coef = setup(cfg)
    g = Box(_dense(cfg), init, coef)
    b = Box(replace(cfg, precision=1), init, coef)
    o = oracle_box(cfg, init)
    got = g.interpyy()
    banded = b.interpyy()
    for f, which, out, ref_b in (("u", 0, got[0], banded[0]), ("w", 0, got[1], banded[1]),
                                 ("v", 1, got[2], banded[2])):
        ref = _oracle_interpyy(cfg, o, o.field(f), which)
        scale = np.abs(ref).max()
        e_dense = np.abs(out - ref).max() / scale
        e_band = np.abs(ref_b - ref).max() / scale
        print(f"{name} interpyy {f}: dense {e_dense:.2e}, banded FP32 {e_band:.2e} (max-abs / max|ref|)")
        assert e_dense <= 2e-6, (f, e_dense)
    g.close()
    b.close()
    o.close()


@pytest.mark.parametrize("name", ["TINY", "C1"])
def test_ydense_one_substep(name):
    cfg = getattr(config, name)
    init, coef = setup(cfg)
    g = Box(_dense(cfg), init, coef)
    b = Box(replace(cfg, precision=1), init, coef)
    o = oracle_box(cfg, init)
    for box in (g, b):
        box.substep(1, True)
    o.substep(1, 1)
    r = _report(f"{name} mixed + dense interpyy, 1 substep", g, o, cfg, coef)
    assert r["vel_rel_l2"] <= 1e-6
    rb = _report(f"{name} mixed + dense interpyy vs banded mixed, 1 substep", g, b, cfg, coef)
    assert rb["vel_rel_l2"] <= 1e-6
    for box in (g, b, o):
        box.close()


def test_ydense_c1_twenty_steps():
    cfg = config.C1
    init, coef = setup(cfg)
    g = Box(_dense(cfg), init, coef)
    o = oracle_box(cfg, init)
    g.advance(20)
    o.advance(20)
    r = _report("C1 mixed + dense interpyy, 20 steps", g, o, cfg, coef)
    assert r["vel_rel_l2"] <= 1e-6
    assert r["max_div"] <= 1e-10
    for k in ("U_rel_l2", "um_rel_l2", "re_theta_rel", "cf_rel"):
        assert r[k] <= 1e-5, k
    g.close()
    o.close()
