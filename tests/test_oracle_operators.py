"""Known-answer tests of the oracle's compact operators (lip.f90) and of the
coefficient restatement (coeft.f90), CPU only.

The reference ships no golden data, so the operators are pinned to the
polynomial degrees that their Pade stencils and boundary closures reproduce
exactly (x: uniform grid, coeft.f90 coef; y: the tanh-stretched grid) and
the coefficient buffer to the closed forms of coeft.f90 and bl_1.F90.
"""
import numpy as np
import pytest

from opentbl_b200 import config, native, synth
from oracle import pyoracle

D = pyoracle.dptr


@pytest.fixture(scope="module")
def tiny():
    cfg = config.TINY
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    ob = pyoracle.OracleBox(cfg, init, threads=1)
    off = native.coef_offsets(cfg)
    yield cfg, init, coef, off, ob
    ob.close()


def _S(coef, off, name):
    return coef[off["SCAL"] + native.SCAL[name]]


def _tol(ref, scale=1.0):
    """Rounding bound: 1e-12 relative to the larger of the result and the
    operator's coefficient scale (1/dy for d/dy, 1/dy^2 for d2/dy2)."""
    return 1e-12 * max(1.0, float(np.abs(ref).max()), scale)


def _dymin(init):
    return float(np.diff(np.asarray(init["y"], dtype=float)).min())


# ---------------- x-lines (pencils (nx, nlin), one line per row here) --------
@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("deg", [0, 1, 2])
def test_interpxx_midpoint_exact(tiny, which, deg):
    """interpxx (lip.f90:248-300) maps values at x_i to x_{i+1/2}; exact for
    quadratics on every row, boundary closures included."""
    cfg, init, coef, off, ob = tiny
    i = np.arange(1, cfg.nx + 1, dtype=float)
    g = np.ascontiguousarray(np.tile(i ** deg, (3, 1)))
    o = np.zeros_like(g)
    ob.L.orc_interpxx(ob.h, D(g), D(o), which, 3)
    ref = (i + 0.5) ** deg
    assert np.abs(o - ref).max() <= _tol(ref)


@pytest.mark.parametrize("which", [0, 1])
def test_interpxx_cubic_interior(tiny, which):
    cfg, init, coef, off, ob = tiny
    i = np.arange(1, cfg.nx + 1, dtype=float)
    g = np.ascontiguousarray(np.tile(i ** 3, (2, 1)))
    o = np.zeros_like(g)
    ob.L.orc_interpxx(ob.h, D(g), D(o), which, 2)
    h = cfg.nx // 2
    ref = (i[:h] + 0.5) ** 3
    assert np.abs(o[:, :h] - ref).max() <= _tol(ref)


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_difvisxx_derivatives_exact(tiny, which, deg):
    """difvisxx (lip.f90:52-142): d/dx of mid-point data onto x_i plus
    rex * d2/dx2 of nodal data, exact for cubics on rows 1..nx-1; row nx is
    the outflow row U_inf*(u_nx - u_{nx-1})*idx (lip.f90:105) with the
    viscous row zeroed (lip.f90:132)."""
    cfg, init, coef, off, ob = tiny
    dx = _S(coef, off, "DX1")
    rex = _S(coef, off, "REX")
    idx = _S(coef, off, "IDX")
    uinf = _S(coef, off, "UINF")
    x = np.arange(1, cfg.nx + 1, dtype=float) * dx
    prod = np.ascontiguousarray(np.tile((x + 0.5 * dx) ** deg, (2, 1)))
    vel = np.ascontiguousarray(np.tile((x / x[-1]) ** deg, (2, 1)))
    out = np.zeros_like(prod)
    ob.L.orc_difvisxx(ob.h, D(prod), D(vel), D(out), which, 2)
    d1 = deg * x ** (deg - 1) if deg else 0 * x
    d2 = deg * (deg - 1) * (x / x[-1]) ** max(deg - 2, 0) / x[-1] ** 2 if deg > 1 else 0 * x
    ref = d1 + rex * d2
    assert np.abs(out[:, :-1] - ref[:-1]).max() <= _tol(ref)
    outflow = uinf * (vel[:, -1] - vel[:, -2]) * idx
    assert np.abs(out[:, -1] - outflow).max() <= _tol(outflow)


# ---------------- y-lines on the stretched grid (one plane) ------------------
def _ypos(cfg, init):
    y = np.asarray(init["y"], dtype=float)   # y(0:ny+1)
    ny = cfg.ny
    return 0.5 * (y[0:ny + 1] + y[1:ny + 2]), y[1:ny + 1]  # u rows 1..ny+1, v rows 1..ny


@pytest.mark.parametrize("deg", [1, 2, 3])
def test_interpyy_u_to_v_exact(tiny, deg):
    """interpyy loguv=0 (lip.f90:359-440): u-type cell values onto the v rows
    with the wall row 1 held at 0 (no slip at y = 0), so it is exact for the
    cubics that vanish at the wall."""
    cfg, init, coef, off, ob = tiny
    yu, yv = _ypos(cfg, init)
    dim = 4
    g = np.ascontiguousarray(np.tile(yu ** deg, (dim, 1)).T)
    o = np.zeros((cfg.ny + 1, dim))
    ob.L.orc_interpyy(ob.h, D(g), D(o), 0, dim, dim)
    ref = yv ** deg
    assert np.abs(o[:cfg.ny] - ref[:, None]).max() <= _tol(ref)


def test_interpyy_v_partition_of_unity(tiny):
    cfg, init, coef, off, ob = tiny
    dim = 3
    g = np.full((cfg.ny, dim), 2.5)
    o = np.zeros((cfg.ny + 1, dim))
    ob.L.orc_interpyy(ob.h, D(g), D(o), 1, dim, dim)
    assert np.abs(o[:cfg.ny] - 2.5).max() <= 1e-13


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_differzy_u_to_v_exact(tiny, deg):
    """differzy v-type (chv=1, lip.f90:152-232): d/dy of u-type cell data onto
    the v rows, exact for cubics on all ny rows."""
    cfg, init, coef, off, ob = tiny
    yu, yv = _ypos(cfg, init)
    nz1 = cfg.nz1
    gi = np.ascontiguousarray(np.tile(yu ** deg, (nz1, 1)).T)
    r = np.zeros((cfg.ny + 1, nz1))
    ob.L.orc_differzy(ob.h, D(gi), D(r), 1)
    ref = deg * yv ** (deg - 1) if deg else 0 * yv
    assert np.abs(r[:cfg.ny] - ref[:, None]).max() <= _tol(ref, 1 / _dymin(init))


@pytest.mark.parametrize("deg", [0, 1])
def test_differzy_v_to_u_exact(tiny, deg):
    cfg, init, coef, off, ob = tiny
    yu, yv = _ypos(cfg, init)
    nz1 = cfg.nz1
    gi = np.zeros((cfg.ny + 1, nz1))
    gi[:cfg.ny] = np.tile(yv ** deg, (nz1, 1)).T
    r = np.zeros((cfg.ny + 1, nz1))
    ob.L.orc_differzy(ob.h, D(np.ascontiguousarray(gi)), D(r), 0)
    ref = deg * yu ** (deg - 1) if deg else 0 * yu
    assert np.abs(r - ref[:, None]).max() <= _tol(ref, 1 / _dymin(init))


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("deg", [0, 1, 2])
def test_vistyy_exact(tiny, which, deg):
    """vistyy (lip.f90:447-513): d2/dy2 on the u rows (which 0) or the v rows
    (which 1), exact for quadratics including the boundary closures."""
    cfg, init, coef, off, ob = tiny
    yu, yv = _ypos(cfg, init)
    src = yu if which == 0 else yv
    jee = len(src)
    u = np.zeros((cfg.ny + 1, cfg.nz1))
    u[:jee] = np.tile(src ** deg, (cfg.nz1, 1)).T
    r = np.zeros((cfg.ny + 1, cfg.nz1))
    ob.L.orc_vistyy(ob.h, D(np.ascontiguousarray(u)), D(r), which)
    ref = deg * (deg - 1) * src ** max(deg - 2, 0) if deg > 1 else 0 * src
    assert np.abs(r[:jee] - ref[:, None]).max() <= _tol(ref, 1 / _dymin(init) ** 2)


@pytest.mark.parametrize("which", [0, 1])
def test_implzy_identity_and_constants(tiny, which):
    """implzy (lip.f90:528-597) solves (A + var1 B) u = A res on rows
    2..jee-1 keeping the boundary rows of u: var1 = 0 returns res; a
    constant res with constant boundary rows is a fixed point for any var1
    (B annihilates constants)."""
    cfg, init, coef, off, ob = tiny
    jee = cfg.ny + 1 if which == 0 else cfg.ny
    rng = np.random.default_rng(7)
    res = np.zeros((cfg.ny + 1, cfg.nz1))
    res[:jee] = rng.standard_normal((jee, cfg.nz1))
    u = res.copy()
    ob.L.orc_implzy(ob.h, D(u), D(np.ascontiguousarray(res)), which, 0.0)
    assert np.abs(u[:jee] - res[:jee]).max() <= 1e-12
    res = np.zeros((cfg.ny + 1, cfg.nz1))
    res[:jee] = 1.75
    u = res.copy()
    ob.L.orc_implzy(ob.h, D(u), D(np.ascontiguousarray(res)), which, -0.37)
    assert np.abs(u[:jee] - 1.75).max() <= 1e-12


# ---------------- coefficient closed forms -----------------------------------
@pytest.mark.parametrize("source", ["oracle", "product"])
@pytest.mark.parametrize("name", ["TINY", "C1", "C2"])
def test_coefficient_closed_forms(name, source):
    cfg = getattr(config, name)
    init = synth.make_initial(cfg)
    y, u0, re, xout = init["y"], init["u0"], init["re"], init["xout"]
    compute = pyoracle.coef_compute if source == "oracle" else native.coef_compute
    coef = compute(cfg, re, xout, y, u0)
    off = native.coef_offsets(cfg)
    S = lambda n: coef[off["SCAL"] + native.SCAL[n]]  # noqa: E731
    nx, nz2 = cfg.nx, cfg.nz2
    # RK3 constants, coeft.f90:494-508
    rk = coef[off["SCAL"] + 20: off["SCAL"] + 32].reshape(4, 3)
    np.testing.assert_array_equal(rk[0], [8 / 15, 5 / 12, 3 / 4])
    np.testing.assert_array_equal(rk[1], [0.0, -17 / 60, -5 / 12])
    np.testing.assert_array_equal(rk[2], [4 / 15, 1 / 15, 1 / 6])
    np.testing.assert_array_equal(rk[3], [4 / 15, 1 / 15, 1 / 6])
    assert S("REX") == -1.0 / S("RE")                       # coeft.f90:480
    assert S("IDX") == 1.0 / S("DX1")                       # coeft.f90:420
    # wavenumbers, bl_1.F90:360-366; kvis = rex*kaz2, coeft.f90:484-486
    k = np.arange(nz2 + 1, dtype=float)
    kaz = coef[off["KAZ"]:off["KAZ"] + nz2 + 1]
    kaz2 = coef[off["KAZ2"]:off["KAZ2"] + nz2 + 1]
    kvis = coef[off["KVIS"]:off["KVIS"] + nz2 + 1]
    # cmplx(0d0, k/az) without KIND is a REAL*4 complex (bl_1.F90:360)
    kz32 = (k / S("AZ")).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(kaz, kz32)
    np.testing.assert_allclose(kaz, k / S("AZ"), rtol=1e-7, atol=0)
    np.testing.assert_array_equal(kaz2, kz32 * kz32)
    np.testing.assert_allclose(kvis, S("REX") * kaz2, rtol=4e-16, atol=0)
    # Poisson eigenvalues in x, coeft.f90:1181-1183
    m = np.arange(1, nx, dtype=float)
    kmod = coef[off["KMOD"]:off["KMOD"] + nx - 1]
    ref = 2.0 / S("DX1") ** 2 * (1 - np.cos(np.pi * (m - 1) / (nx - 1)))
    np.testing.assert_allclose(kmod, ref, rtol=1e-14, atol=1e-14 * ref.max())
    # y metrics: idyy(j) = 2/(dy(j-1)+dy(j)), coeft.f90:424
    dy = coef[off["DY"]:off["DY"] + cfg.ny + 1]
    idyy = coef[off["IDYY"]:off["IDYY"] + cfg.ny]
    np.testing.assert_allclose(idyy, 2.0 / (dy[:-1] + dy[1:]), rtol=1e-15)
    # packed buffer is deterministic
    np.testing.assert_array_equal(coef, compute(cfg, re, xout, y, u0))
