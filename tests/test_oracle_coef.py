"""The coefficient set-up (coeft.f90 coef, bl_1.F90 wavenumbers and
inlet_retheta, boun.f90 magicnumber), CPU only.

Two separate restatements compute the packed buffer: the product's
otbl_coef_compute (opentbl_b200/csrc/coef.cpp) and the oracle's
orc_coef_compute (oracle/orc_coef.c). They must agree bit for bit on every
box the tests, the bench and the ensemble use. Quantities that no stencil
exactness test pins are checked here against numpy restatements of their
definitions: vmagic (boun.f90:114-140), rthin and din (bl_1.F90:380-388),
the zero-vorticity closures ccon (coeft.f90:901-924 via coefb flags 6 and
7), the y-Poisson operator ayp (mtr, coeft.f90:1244-1332) and the
single-precision wavenumbers kaz (bl_1.F90:360).
"""
import numpy as np
import pytest

from opentbl_b200 import config, ensemble, native, synth
from oracle import pyoracle

BOXES = [config.TINY, config.SMALL, config.C1, config.C2, config.MED, config.SLAB,
         config.replace(config.C1, xpose_round=1), config.replace(config.C2, precision=1)]
BOXES += ensemble.ensemble_configs(24)


def _both(cfg):
    init = synth.make_initial(cfg)
    args = (cfg, init["re"], init["xout"], init["y"], init["u0"])
    return init, native.coef_compute(*args), pyoracle.coef_compute(*args)


def _arr(coef, cfg, name):
    off = native.coef_offsets(cfg)
    names = native.COEF_NAMES + ("TOTAL",)
    i = names.index(name)
    return coef[off[name]:off[names[i + 1]]]


def _scal(coef, cfg, name):
    return _arr(coef, cfg, "SCAL")[native.SCAL[name]]


@pytest.mark.parametrize("cfg", BOXES, ids=lambda c: c.name + ("-r4" if c.xpose_round else "")
                         + ("-mixed" if c.precision else ""))
def test_product_and_oracle_bitwise(cfg):
    _, a, b = _both(cfg)
    assert len(a) == len(b) == pyoracle.coef_count(cfg)
    if not np.array_equal(a, b):
        bad = [n for n in native.COEF_NAMES
               if not np.array_equal(_arr(a, cfg, n), _arr(b, cfg, n))]
        raise AssertionError(f"coefficient arrays differ: {bad}")


@pytest.fixture(scope="module", params=["TINY", "C1", "C2"])
def box(request):
    cfg = getattr(config, request.param)
    init, _, coef = _both(cfg)
    return cfg, init, coef


def test_kaz_single_precision(box):
    """kaz(k) = cmplx(0d0, k/az) is a default (REAL*4) complex; kaz2 = -kaz**2."""
    cfg, init, coef = box
    az = _scal(coef, cfg, "AZ")
    k = np.arange(cfg.nz2 + 1, dtype=np.float64)
    s = (k / az).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_arr(coef, cfg, "KAZ"), s)
    np.testing.assert_array_equal(_arr(coef, cfg, "KAZ2"), s * s)
    np.testing.assert_array_equal(_arr(coef, cfg, "KVIS"), _scal(coef, cfg, "REX") * (s * s))


def test_inlet_retheta(box):
    """bl_1.F90:380-388: U_inf from 16 points below the top, delta99 where
    u0 first reaches 0.99 U_inf (REAL*4 literal), theta by the rectangle sum."""
    cfg, init, coef = box
    ny = cfg.ny
    u0 = np.asarray(init["u0"], dtype=np.float64)    # u0(1:ny+1) at [j-1]
    y = np.asarray(init["y"], dtype=np.float64)      # y(0:ny+1) at [j]
    dy = np.diff(y)                                  # dy(0:ny) at [j]
    uinf = u0[ny - 20:ny - 4].sum() / 16.0           # u0(ny+1-20 : ny+1-5)
    u99 = float(np.float32(0.99)) * uinf
    hits = [j for j in range(1, ny - 1) if u0[j - 1] >= u99]
    jtop = hits[0] if hits else ny - 1
    din = y[jtop]
    k = np.arange(2, jtop + 4)                       # u0(2:jtop+3), dy(1:jtop+2)
    rthin = np.sum((uinf - u0[k - 1]) * u0[k - 1] * dy[k - 1]) * cfg_re(init) / uinf
    assert _scal(coef, cfg, "DIN") == din
    np.testing.assert_allclose(_scal(coef, cfg, "RTHIN"), rthin, rtol=1e-13)
    # the synthetic inlet profile was built for this Re_theta
    np.testing.assert_allclose(_scal(coef, cfg, "RTHIN"), cfg.re_theta, rtol=0.05)


def cfg_re(init):
    return float(init["re"])


def test_vmagic(box):
    """boun.f90:114-140: delta*(x) from the Nagib-Chauhan-Monkewitz fits and
    its centred derivative on x = (i-1)*ax*pi/(nx-1)."""
    cfg, init, coef = box
    nx = cfg.nx
    re = _scal(coef, cfg, "RE")
    rthin = _scal(coef, cfg, "RTHIN")
    e1, c1, kap, ckap, cprim = 0.8659, 0.01277, 0.384, 4.127, 7.135
    x = np.arange(nx) * (_scal(coef, cfg, "AX") * np.pi / (nx - 1))
    reth = (rthin ** (1 / e1) + c1 ** (1 / e1) * re * x) ** e1
    uep = np.log(reth) / kap + ckap
    h = reth / ((1 - cprim / uep) * re)
    ref = np.empty(nx)
    ref[0] = (h[1] - h[0]) / (x[1] - x[0])
    ref[1:-1] = (h[2:] - h[:-2]) / (x[2:] - x[:-2])
    ref[-1] = (h[-1] - h[-2]) / (x[-1] - x[-2])
    got = _arr(coef, cfg, "VMAGIC")
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
    assert np.all(got > 0)  # delta* grows downstream: the top sucks fluid out


def test_ayp_second_difference(box):
    """mtr: row j of ayp is (1/h_j) [2 (phi_{j+1}-phi_j)/(h_j+h_{j+1})
    - 2 (phi_j-phi_{j-1})/(h_{j-1}+h_j)], h_j = y(j+1)-y(j), with zero
    gradient at both ends (rows 1 and ny-1)."""
    cfg, init, coef = box
    ny = cfg.ny
    y = _arr(coef, cfg, "Y")
    h = np.diff(y)                                   # h[j] = y(j+1)-y(j), j = 0..ny
    ayp = _arr(coef, cfg, "AYP").reshape(ny, 3)[:ny - 1]   # rows j = 1..ny-1
    for j in range(1, ny):
        gm = 0.0 if j == 1 else 2.0 / (h[j - 1] + h[j])
        gp = 0.0 if j == ny - 1 else 2.0 / (h[j] + h[j + 1])
        ref = np.array([gm, -(gm + gp), gp]) / h[j]
        np.testing.assert_allclose(ayp[j - 1], ref, rtol=1e-13, atol=0)
    # constants are in its null space (Neumann at the wall and the top)
    rows = ayp.sum(axis=1)
    assert np.abs(rows).max() <= 1e-12 * np.abs(ayp).max()


def _moments(pos, rows, quirk_rows34=False):
    """Moment matrix of a one-sided stencil at offsets pos: row r is
    pos**r / r! (r = 0..rows-1)."""
    M = np.array([[p ** r / float(np.prod(np.arange(1, r + 1))) for p in pos]
                  for r in range(rows)])
    if quirk_rows34:
        M[2, 2:] *= 2.0
    return M


def test_ccon_zero_vorticity_closures(box):
    """ccon rows: first-derivative stencils that define the ghost rows of u
    and w (boun.f90:7-56). Row 1 (coefb flag 7, coeft.f90:901-911) at
    offsets (a/2, -b/2, -(b/2+c), -(b/2+c+d)) with the reference's second
    moment of the last two points missing its 1/2 (coeft.f90:1657-1658);
    row 2 (flag 6, :913-922) at (0, -a/2, -(a/2+b), -(a/2+b+c)). Both solve
    M c = e_2 (moments 0..3)."""
    cfg, init, coef = box
    ny = cfg.ny
    y = _arr(coef, cfg, "Y")
    dy = np.diff(y)
    dyi = np.zeros(ny + 1)
    dyi[1:] = 0.5 * (dy[1:] + dy[:-1])
    ccon = _arr(coef, cfg, "CCON").reshape(4, 2).T       # ccon(r, c) column-major
    a, b, c, d = dy[ny], dy[ny - 1], dyi[ny - 1], dyi[ny - 2]
    pos7 = [a / 2, -b / 2, -(b / 2 + c), -(b / 2 + c + d)]
    a6, b6, c6 = -dy[0], -dyi[1], -dyi[2]
    pos6 = [0.0, -a6 / 2, -(a6 / 2 + b6), -(a6 / 2 + b6 + c6)]
    for row, M in ((ccon[0], _moments(pos7, 4, quirk_rows34=True)), (ccon[1], _moments(pos6, 4))):
        e2 = np.array([0.0, 1.0, 0.0, 0.0])
        resid = M @ row - e2
        scale = np.abs(M) @ np.abs(row)
        assert np.all(np.abs(resid) <= 1e-11 * np.maximum(scale, 1.0)), (resid, scale)
        np.testing.assert_allclose(row, np.linalg.solve(M, e2), rtol=1e-7, atol=0)
