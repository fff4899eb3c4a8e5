"""Properties of the oracle's substep (CPU only): the projection leaves a
divergence-free field, the integral quantities of genflu agree with an
independent numpy restatement of genflu.F90:67-93, the REAL4 transpose mode
perturbs the FP64 result at single-precision level only, the fixed-dt mode
holds dt, and the result does not depend on the thread count."""
import ctypes

import numpy as np
import pytest

from opentbl_b200 import config, native, synth
from opentbl_b200.config import replace
from oracle import pyoracle

from helpers import oracle_box, rel_l2, setup

STATE = ("u", "v", "w", "p", "rhsupa", "rhsvpa", "rhswpa")


@pytest.fixture(scope="module")
def tiny():
    return setup(config.TINY)


def test_projection_is_divergence_free(tiny):
    """pois.f90:11-239: after rhsp + outflow_correction + pois the
    divergence of pois.f90:41-54 is at round-off."""
    init, coef = tiny
    ob = oracle_box(config.TINY, init, threads=2)
    d0 = np.abs(ob.divergence()).max()
    ob.substep(1, 1)
    d1 = np.abs(ob.divergence()).max()
    ob.substep(2, 0)
    ob.substep(3, 0)
    d3 = np.abs(ob.divergence()).max()
    assert d1 <= 1e-11 and d3 <= 1e-12, (d0, d1, d3)


def _genflu_numpy(ucol0, um, y, dy, re, rthin, dt, tloc):
    """genflu.F90:67-93 on plane-1 mode-0 u (rows 1..ny+1), numpy."""
    ny = len(um) - 1
    timec = 20.0 if tloc < 20 else (100.0 if tloc < 100 else tloc)
    a = dt / timec
    um = a * ucol0 + um * (1.0 - a)
    U = np.concatenate([[np.nan], um])              # 1-based
    utau = np.sqrt(abs((U[2] - U[1]) / (y[2] - y[1]) / re))
    uinf = U[ny + 1 - 20:ny + 1 - 5 + 1].sum() / 16.0
    u99 = float(np.float32(0.99)) * uinf
    jtop = 0
    for j in range(1, ny - 1):
        if U[j] >= u99:
            break
        jtop = j + 1
    dout = y[jtop]
    q = np.arange(jtop + 2)
    rth = ((uinf - U[2 + q]) * U[2 + q] * dy[1 + q]).sum() * re / uinf
    g2 = rthin / rth
    return um, dict(timec=timec, utauout=utau, dout=dout, rthout=rth, gamma2=g2, gamma1=g2 ** 0.125)


@pytest.mark.parametrize("tiempo", [3.0, 50.0, 250.0])
def test_genflu_integrals_against_numpy(tiny, tiempo):
    init, coef = tiny
    cfg = config.TINY
    ob = oracle_box(cfg, init, threads=1)
    st = pyoracle.OtblInflow()
    st.dt, st.tiempo, st.timeinit = 0.05, tiempo, 0.0
    um0 = np.ascontiguousarray(init["um"])
    ob.L.orc_set_inflow(ob.h, pyoracle.dptr(np.ascontiguousarray(init["u0"])),
                        pyoracle.dptr(np.ascontiguousarray(init["v0"])), pyoracle.dptr(um0),
                        ctypes.byref(st))
    xout = int(init["xout"])
    ucol = ob.field("u")[xout - 1, :, 0].copy()
    ob.L.orc_genflu(ob.h)
    um, got = ob.inflow()
    off = native.coef_offsets(cfg)
    y = coef[off["Y"]:off["Y"] + cfg.ny + 2]
    dy = coef[off["DY"]:off["DY"] + cfg.ny + 1]
    S = coef[off["SCAL"]:]
    um_ref, ref = _genflu_numpy(ucol, um0, y, dy, S[native.SCAL["RE"]], S[native.SCAL["RTHIN"]],
                                0.05, tiempo)
    assert rel_l2(um, um_ref) <= 1e-15
    for k, v in ref.items():
        assert abs(got[k] - v) <= 1e-13 * max(1.0, abs(v)), (k, got[k], v)
    # plane 1 after recycling: modes 0 are the inlet profiles (genflu.F90:146-150)
    u = ob.field("u")
    assert np.array_equal(u[0, :, 0], np.asarray(init["u0"], dtype=float))
    assert np.all(u[0, :, 1] == 0.0)


def _energies_numpy(cfg, coef, u, v, w):
    """energies/ministats (rhsp.F90:493-509, stotf.F90:395-440) for one
    domain: plane nx/2's branch, which overwrites plane 1's ener(1:3); then
    ener(13:15) = 0 (rhsp.F90:487)."""
    o = native.coef_offsets(cfg)
    hy = coef[o["HY"]:o["HY"] + cfg.ny + 1]
    i = cfg.nx // 2 - 1
    e = np.zeros(15)
    for f, g in enumerate((u[i], v[i], w[i])):
        c = g[:, 0::2] + 1j * g[:, 1::2]
        aux = 2.0 * (np.abs(c[:, 1:]) ** 2).sum(axis=1) + c[0, 0].real ** 2
        e[f] = (aux * hy[:len(aux)]).sum()
        e[3 + 4 * f:7 + 4 * f] = (c[0, 0].real, c[1, 0].real,
                                  aux[0] - c[0, 0].real ** 2, aux[1] - c[0, 0].real ** 2)
    e[12:] = 0.0
    return e


def test_energies_against_numpy(tiny):
    """ener after rhsp(m=1) is computed from the state rhsp was called on;
    substeps 2 and 3 leave it alone."""
    init, coef = tiny
    ob = oracle_box(config.TINY, init, threads=2)
    assert not ob.energies().any()
    u, v, w = (ob.field(n).copy() for n in "uvw")
    ob.substep(1, 1)
    e = ob.energies()
    ref = _energies_numpy(config.TINY, coef, u, v, w)
    assert np.allclose(e, ref, rtol=1e-13, atol=0.0), (e, ref)
    assert e[0] > 0 and e[1] > 0 and e[2] > 0
    ob.substep(2, 0)
    assert np.array_equal(ob.energies(), e)


def test_real4_transposes_perturb_at_single_precision(tiny):
    init, coef = tiny
    a = oracle_box(config.TINY, init, threads=1)
    b = oracle_box(replace(config.TINY, xpose_round=1), init, threads=1)
    a.substep(1, 1)
    b.substep(1, 1)
    e = [rel_l2(b.field(n), a.field(n)) for n in ("u", "v", "w")]
    assert max(e) <= 1e-6 and min(e) > 0.0, e


def test_fixed_dt_mode(tiny):
    init, coef = tiny
    cfg = replace(config.TINY, dt_mode=1, dt_fixed=0.0125)
    ob = oracle_box(cfg, init, threads=1)
    ob.advance(2)
    um, st = ob.inflow()
    assert st["dt"] == 0.0125
    assert abs(st["tiempo"] - 2 * 0.0125) <= 1e-16


def test_adaptive_dt_is_the_cfl_limit(tiny):
    """rhsp.F90:214-262: dt = min(dxmin/umax, dzmin/wmax, min_j dymin_j/vm_j,
    dtret); with the maxima reported by the oracle the limit is reproduced."""
    init, coef = tiny
    cfg = config.TINY
    ob = oracle_box(cfg, init, threads=1)
    ob.rhsp(1, 1)
    um, st = ob.inflow()
    off = native.coef_offsets(cfg)
    S = coef[off["SCAL"]:]
    dt = st["dt"]
    assert dt > 0 and np.isfinite(dt)
    assert dt <= S[native.SCAL["DXMIN"]] / st["umax"] * (1 + 1e-15)
    assert dt <= S[native.SCAL["DZMIN"]] / st["wmax"] * (1 + 1e-15)
    assert dt <= S[native.SCAL["DTRET"]] * (1 + 1e-15)


def test_threads_do_not_change_the_result(tiny):
    init, coef = tiny
    res = []
    for t in (1, 4):
        ob = oracle_box(config.TINY, init, threads=t)
        ob.advance(1)
        res.append({n: ob.field(n) for n in STATE})
        ob.close()
    for n in STATE:
        assert rel_l2(res[1][n], res[0][n]) <= 1e-14, n


def test_synthetic_fields_are_seeded():
    a = synth.make_initial(config.TINY)
    b = synth.make_initial(config.TINY)
    c = synth.make_initial(replace(config.TINY, seed=99))
    for n in ("u", "v", "w"):
        assert np.array_equal(a[n], b[n])
        assert not np.array_equal(a[n], c[n])
        assert np.isfinite(a[n]).all()
    # mean profile: 0 at the wall row of v-type, free stream 1 at the top
    assert abs(a["u0"][-1] - 1.0) <= 1e-12
