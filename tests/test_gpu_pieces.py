"""The standalone pieces of the path on caller-owned device buffers, each
against the oracle's counterpart on the same input:

  otbl_chp2x / otbl_chx2p  change.f90:224-275 (planes <-> pencils, with and
                           without the REAL*4 rounding of change.f90:579,608)
  otbl_fourxz              ffts.f90:27-67 (r2c with 1/nz and 2/3 truncation;
                           c2r with the modes above nz2 zeroed)
  otbl_cosftx              ffts.f90:147-181 (REDFT10 x 1/(nx-1), REDFT01 x 0.5)
  otbl_boun                boun.f90:7-56 (on the context's own state)

The transposes are pure permutations (bit for bit, in both rounding modes);
the transforms agree to FP64 rounding (1e-13 relative L2).
"""
import numpy as np
import pytest

from opentbl_b200 import Box, config
from opentbl_b200.config import replace
from oracle import pyoracle

from helpers import oracle_box, rel_l2, setup

pytestmark = pytest.mark.gpu

D = pyoracle.dptr


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _pair(cfg):
    init, coef = setup(cfg)
    return Box(cfg, init, coef), oracle_box(cfg, init, threads=4), init


@pytest.mark.parametrize("xr", [0, 1], ids=["fp64", "real4"])
@pytest.mark.parametrize("utype", [True, False], ids=["jee=ny+1", "jee=ny"])
def test_chp2x_chx2p(xr, utype):
    torch = pytest.importorskip("torch")
    cfg = replace(config.SMALL, xpose_round=xr)
    g, o, _ = _pair(cfg)
    jee = cfg.ny + 1 if utype else cfg.ny
    rng = np.random.default_rng(5)
    plan = rng.standard_normal((cfg.nx, jee, cfg.nz1))
    pen_o = np.zeros((cfg.nz1 * jee, cfg.nx))
    o.L.orc_chp2x(o.h, D(pen_o), D(plan), jee)
    dplan = _dev(torch, plan)
    dpen = torch.zeros((cfg.nz1 * jee, cfg.nx), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.chp2x(dpen.data_ptr(), dplan.data_ptr(), jee)
    g.sync()
    pen_g = dpen.cpu().numpy()
    np.testing.assert_array_equal(pen_g, pen_o)
    if xr:
        assert np.array_equal(pen_g, pen_g.astype(np.float32).astype(np.float64))
    else:
        np.testing.assert_array_equal(pen_g, plan.reshape(cfg.nx, -1).T)
    # and back: pencils -> planes
    pen = rng.standard_normal((cfg.nz1 * jee, cfg.nx))
    plan_o = np.zeros((cfg.nx, jee, cfg.nz1))
    o.L.orc_chx2p(o.h, D(pen), D(plan_o), jee)
    dpen = _dev(torch, pen)
    dplan = torch.zeros((cfg.nx, jee, cfg.nz1), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.chx2p(dpen.data_ptr(), dplan.data_ptr(), jee)
    g.sync()
    np.testing.assert_array_equal(dplan.cpu().numpy(), plan_o)


@pytest.mark.parametrize("nz", [32, 64, 128, 256, 512])
def test_fourxz(nz):
    torch = pytest.importorskip("torch")
    cfg = replace(config.TINY, nz=nz, name=f"tiny-nz{nz}")
    g, o, _ = _pair(cfg)
    nlines = 77
    rng = np.random.default_rng(nz)
    # r2c: physical lines (nz reals and two pad slots) -> modes 0..nz2
    phys = np.zeros((nlines, nz + 2))
    phys[:, :nz] = rng.standard_normal((nlines, nz))
    fou_o = np.zeros((nlines, cfg.nz1))
    o.L.orc_fourxz(o.h, D(fou_o), D(phys.copy()), -1, nlines)
    dphys = _dev(torch, phys)
    dfou = torch.zeros((nlines, cfg.nz1), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.fourxz(dfou.data_ptr(), dphys.data_ptr(), -1, nlines)
    g.sync()
    assert rel_l2(dfou.cpu().numpy(), fou_o) <= 1e-13
    # c2r: modes -> physical lines
    fou = rng.standard_normal((nlines, cfg.nz1))
    fou[:, 1] = 0.0  # mode 0 is real
    phys_o = np.zeros((nlines, nz + 2))
    o.L.orc_fourxz(o.h, D(fou.copy()), D(phys_o), 1, nlines)
    dfou = _dev(torch, fou)
    dphys = torch.zeros((nlines, nz + 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.fourxz(dfou.data_ptr(), dphys.data_ptr(), 1, nlines)
    g.sync()
    got = dphys.cpu().numpy()
    assert rel_l2(got[:, :nz], phys_o[:, :nz]) <= 1e-13
    # round trip through the GPU alone: r2c(c2r(f)) = f / 1 on modes 0..nz2
    dfou2 = torch.zeros_like(dfou)
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.fourxz(dfou2.data_ptr(), dphys.data_ptr(), -1, nlines)
    g.sync()
    assert rel_l2(dfou2.cpu().numpy(), fou) <= 1e-13


@pytest.mark.parametrize("nx", [33, 65, 257, 385, 1025])
@pytest.mark.parametrize("iopt", [-1, 1], ids=["redft10", "redft01"])
def test_cosftx(nx, iopt):
    torch = pytest.importorskip("torch")
    cfg = replace(config.TINY, nx=nx, name=f"tiny-nx{nx}")
    g, o, _ = _pair(cfg)
    nlines = 13
    rng = np.random.default_rng(nx)
    c = rng.standard_normal((nlines, nx))
    c_o = c.copy()
    o.L.orc_cosftx(o.h, D(c_o), nlines, iopt)
    dc = _dev(torch, c)
    torch.cuda.synchronize()  # buffers were filled on torch's stream
    g.cosftx(dc.data_ptr(), nlines, iopt)
    g.sync()
    got = dc.cpu().numpy()
    np.testing.assert_array_equal(got[:, 0], c[:, 0])  # element 1 is not transformed
    assert rel_l2(got, c_o) <= 1e-13


def test_boun():
    """boun on a random state: v rows 1 and ny (with vmagic on mode 0 of row
    ny), the ghost rows 1 and ny+1 of u and w from inby and ccon."""
    cfg = config.SMALL
    g, o, init = _pair(cfg)
    rng = np.random.default_rng(9)
    for n in ("u", "v", "w"):
        a = rng.standard_normal(g.shape(n))
        g.set_field(n, a)
        o.set_field(n, a)
    g.boun()
    o.L.orc_boun(o.h)
    for n in ("u", "v", "w"):
        assert rel_l2(g.field(n), o.field(n)) <= 1e-15, n
    v = g.field("v")
    assert not v[:, 0, :].any()
    np.testing.assert_array_equal(v[:, cfg.ny - 1, 1:], 0.0)
