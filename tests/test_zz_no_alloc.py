"""otbl_genflu_noalloc (genflu on caller-owned device buffers, scratch plane
in a static device array) against otbl_genflu on the same state, two calls in
a row. Collected last so that it also runs after every other GPU test in the
same process; it passes alone as well."""
import ctypes

import numpy as np
import pytest

from opentbl_b200 import Box, config, native
from opentbl_b200.config import replace

from helpers import rel_l2, setup

pytestmark = pytest.mark.gpu

# include/otbl.h: scal slots and the static scratch size
GF_DT, GF_TIEMPO, GF_TIMEINIT, GF_TIMEC, GF_UTAUOUT, GF_RTHOUT, GF_DOUT, GF_GAMMA1, GF_GAMMA2, GF_COUNT = range(10)
SCRATCH_MAX = 2048
OUT_SLOTS = {"timec": GF_TIMEC, "utauout": GF_UTAUOUT, "rthout": GF_RTHOUT, "dout": GF_DOUT,
             "gamma1": GF_GAMMA1, "gamma2": GF_GAMMA2}


def _bind(L):
    f = L.otbl_genflu_noalloc
    f.argtypes = [ctypes.c_void_p] * 9
    f.restype = ctypes.c_int
    return f


def _dev(torch, a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype or np.float64)).to("cuda:0")


def _noalloc_call(fn, box, bufs):
    return fn(box.h, *(t.data_ptr() for t in (bufs["u"], bufs["v"], bufs["w"], bufs["u0"], bufs["v0"],
                                                bufs["um"], bufs["scal"], bufs["err"])))


def test_genflu_noalloc_matches_genflu_two_calls():
    torch = pytest.importorskip("torch")
    cfg = config.SMALL
    assert 3 * (cfg.ny + 1) + 2 <= SCRATCH_MAX
    init, coef = setup(cfg)
    g = Box(cfg, init, coef)
    fn = _bind(g.L)
    dt, tiempo, timeinit = 0.05, 3.0, 0.0
    inf = native.OtblInflow()
    inf.dt, inf.tiempo, inf.timeinit = dt, tiempo, timeinit
    u0 = np.ascontiguousarray(init["u0"], dtype=np.float64)
    v0 = np.ascontiguousarray(init["v0"], dtype=np.float64)
    um = np.ascontiguousarray(init["um"], dtype=np.float64)
    assert g.L.otbl_set_inflow(g.h, native.dptr(u0), native.dptr(v0), native.dptr(um), ctypes.byref(inf)) == 0
    scal = np.zeros(GF_COUNT)
    scal[[GF_DT, GF_TIEMPO, GF_TIMEINIT]] = dt, tiempo, timeinit
    bufs = {n: _dev(torch, init[n]) for n in ("u", "v", "w")}
    bufs.update(u0=_dev(torch, u0), v0=_dev(torch, v0[:cfg.ny]), um=_dev(torch, um), scal=_dev(torch, scal),
                err=_dev(torch, np.zeros(1), np.int32))
    torch.cuda.synchronize()
    for call in range(2):
        g.genflu()
        assert _noalloc_call(fn, g, bufs) == 0, g.L.otbl_last_error(g.h)
        g.sync()
        torch.cuda.synchronize()
        for n in ("u", "v", "w"):
            mine = bufs[n].cpu().numpy().reshape(g.shape(n))
            ref = g.field(n)
            assert rel_l2(mine[0], ref[0]) <= 1e-13, (call, n)
            assert np.array_equal(mine[1:], ref[1:]), (call, n)
        um_ref, st = g.inflow()
        assert rel_l2(bufs["um"].cpu().numpy(), um_ref) <= 1e-15, call
        s = bufs["scal"].cpu().numpy()
        for k, slot in OUT_SLOTS.items():
            assert abs(s[slot] - st[k]) <= 1e-13 * max(1.0, abs(st[k])), (call, k, s[slot], st[k])
        assert int(bufs["err"].cpu()[0]) == 0


@pytest.mark.parametrize("ny", [681, 700])
def test_genflu_noalloc_rejects_oversized_plane_and_nulls(ny):
    """ny = 681 still fits the tables (3*682+2 = 2048 doubles) but not 48 KB
    of shared memory; ny = 700 fits neither. Both are refused before any
    launch."""
    torch = pytest.importorskip("torch")
    big = replace(config.SMALL, nx=9, ny=ny, nz=32, name=f"tall-9x{ny}x32")
    assert 3 * (big.ny + 1) + 2 > SCRATCH_MAX or ny == 681
    init, coef = setup(big)
    g = Box(big, init, coef)
    fn = _bind(g.L)
    bufs = {n: _dev(torch, np.zeros(8)) for n in ("u", "v", "w", "u0", "v0", "um", "scal")}
    bufs["err"] = _dev(torch, np.zeros(1), np.int32)
    torch.cuda.synchronize()
    launches = g.launches
    assert _noalloc_call(fn, g, bufs) == 2  # OTBL_ERR_CONFIG
    assert b"OTBL_GENFLU_SCRATCH_MAX" in g.L.otbl_last_error(g.h)
    assert g.launches == launches
    small = Box(config.TINY, *setup(config.TINY))
    assert fn(small.h, None, None, None, None, None, None, None, None) == 1  # OTBL_ERR_ARG
