"""Known-answer tests of the oracle's one-point statistics (statsp,
stotf.F90:51-291) and of its compact operators (lip.f90:666-809 with the
fd_* coefficients of coeft.f90:56-318), CPU only.

The operators are pinned to the polynomial degrees their stencils and
closures reproduce (measured: diffx degree 5, interpx_new 4 on the uniform
x grid; on the stretched y grid interpy_new 4 for u and w, 3 for p, diffy
4), and statsp to a mean flow whose statistics follow in closed form.
"""
import numpy as np
import pytest

from opentbl_b200 import config, native, synth
from oracle import pyoracle

ST = {n: i for i, n in enumerate(
    "ua va wa pm dudx0 dvdx0 dwdx0 dudy0 dvdy0 dwdy0 vortxa vortya vortza us vs ws uv uw vw "
    "pup pvp pp pdudx pdudy pdvdx pdvdy pdwdz vortx vorty vortz dispu dispv dispw dispuv "
    "u3 v3 u2v v2u w2v w2u".split())}


def test_stat_indices_match_header():
    import re
    import os
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "otbl.h")).read()
    start = hdr.index("OTBL_ST_UA = 0")
    block = hdr[start:hdr.index("OTBL_NSTATS", start)]
    names = [m.lower() for m in re.findall(r"OTBL_ST_(\w+)", block)]
    assert names == list(ST), names
    assert pyoracle.OracleBox.NSTATS == len(ST) == 40


@pytest.fixture(scope="module", params=["TINY", "C1"])
def box(request):
    cfg = getattr(config, request.param)
    init = synth.make_initial(cfg)
    ob = pyoracle.OracleBox(cfg, init, threads=2)
    yield cfg, init, ob
    ob.close()


def _grids(cfg, init):
    y = np.asarray(init["y"], dtype=float)            # y(0:ny+1), y(1) = 0 at the wall
    yp = 0.5 * (y[0:cfg.ny + 1] + y[1:cfg.ny + 2])      # u rows yp(1:ny+1)
    dx = cfg.ax * np.pi / (cfg.nx + 1)
    x = np.arange(1, cfg.nx + 1) * dx
    return y, yp, dx, x


@pytest.mark.parametrize("deg", range(0, 6))
def test_x_operators_exact(box, deg):
    cfg, init, ob = box
    y, yp, dx, x = _grids(cfg, init)
    L = x.max()
    f = (x / L) ** deg
    d = ob.stats_operator(1, f, cfg.nx)
    ref = deg * (x / L) ** max(deg - 1, 0) / L if deg else 0 * x
    assert np.abs(d - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    if deg <= 4:
        o = ob.stats_operator(0, f, cfg.nx)
        assert np.abs(o - ((x + dx / 2) / L) ** deg).max() <= 1e-12


@pytest.mark.parametrize("deg", range(1, 5))
def test_y_operators_exact(box, deg):
    cfg, init, ob = box
    y, yp, dx, x = _grids(cfg, init)
    ny, H = cfg.ny, y[cfg.ny]
    ref = (y[1:ny + 1] / H) ** deg
    # u and w: wall row held at 0 (no slip), so polynomials that vanish there
    o = ob.stats_operator(2, (yp / H) ** deg, ny)
    assert np.abs(o - ref).max() <= 1e-12
    if deg <= 3:
        o = ob.stats_operator(3, (yp[:ny] / H) ** deg, ny)   # p, extrapolated to the wall
        assert np.abs(o - ref).max() <= 1e-12
    o = ob.stats_operator(4, ref, ny)
    dref = deg * (y[1:ny + 1] / H) ** (deg - 1) / H
    assert np.abs(o - dref).max() <= 1e-12 * max(1.0, np.abs(dref).max())


def test_statsp_mean_flow_closed_form(box):
    """u = U(y) = (y/H)^2 in mode 0 of every plane, v = w = p = 0: every
    statistic follows from U and dU/dy (the x operators are exact on
    constants, interpy_new and diffy on quadratics)."""
    cfg, init, ob = box
    y, yp, dx, x = _grids(cfg, init)
    ny, nx, H = cfg.ny, cfg.nx, y[cfg.ny]
    for f in ("u", "v", "w", "p"):
        ob.set_field(f, np.zeros_like(ob.field(f)))
    u = np.zeros((nx, ny + 1, cfg.nz1))
    u[:, :, 0] = (yp / H) ** 2
    ob.set_field("u", u)
    acc = ob.statsp()
    U = (y[1:ny + 1] / H) ** 2
    dU = 2 * y[1:ny + 1] / H ** 2
    exp = {"ua": U, "us": U * U, "u3": cfg.nz * U ** 3, "dudy0": dU, "vortza": -dU,
           "dispu": dU * dU, "vorty": 0 * U, "vortz": dU * dU}
    for name, ref in exp.items():
        got = acc[ST[name]]
        assert np.abs(got - ref[None, :]).max() <= 1e-11 * max(1.0, np.abs(ref).max()), name
    for name in ("va", "wa", "pm", "vs", "ws", "uv", "uw", "vw", "pp", "v3", "w2u", "u2v",
                 "dudx0", "dvdx0", "dwdx0", "dvdy0", "dwdy0", "vortxa", "vortya", "dispv", "dispw"):
        assert np.abs(acc[ST[name]]).max() <= 1e-11, name
    # one statsp call is one sample: a second call adds the same again
    acc2 = ob.statsp(acc.copy())
    assert np.allclose(acc2, 2 * acc, rtol=1e-14, atol=0)


def test_statsp_seeded_field_symmetries(box):
    """On the seeded field: Reynolds stresses and the Parseval-weighted
    energies are non-negative, and the k = 0 part of us is ua^2."""
    cfg, init, ob = box
    for f in ("u", "v", "w", "p"):
        ob.set_field(f, init[f])
    acc = ob.statsp()
    for name in ("us", "vs", "ws", "pp", "vortx", "vorty", "vortz", "dispu", "dispv", "dispw"):
        assert acc[ST[name]].min() >= 0.0, name
    assert np.all(acc[ST["us"]] >= acc[ST["ua"]] ** 2 * (1 - 1e-12))
