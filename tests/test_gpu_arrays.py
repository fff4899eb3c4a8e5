"""The reference's array surface (otbl_bind_state and the *_arrays entry
points of include/otbl.h: rhsp.F90:22-27, boun.f90:7,63, pois.f90:11,
genflu.F90:3) on caller-owned device arrays, bit for bit against the
context API on the same input."""
import ctypes

import numpy as np
import pytest

from opentbl_b200 import Box, config, native
from opentbl_b200.config import replace

from helpers import setup

pytestmark = pytest.mark.gpu

FIELDS = native.FIELDS


def _caller_arrays(torch, init):
    arr = {n: torch.from_numpy(np.ascontiguousarray(init[n], dtype=np.float64)).cuda() for n in FIELDS}
    torch.cuda.synchronize()  # filled on torch's stream; the library uses its own
    return arr


def _same(torch, box, arr):
    torch.cuda.synchronize()
    for n in FIELDS:
        got = arr[n].cpu().numpy()
        ref = box.field(n)
        assert np.array_equal(got, ref), (n, float(np.abs(got - ref).max()))


@pytest.mark.parametrize("name", ["TINY", "SMALL"])
def test_substeps_on_caller_arrays(name):
    """One RK3 step (bl_1.F90:94-125) through rhsp_arrays,
    outflow_correction_arrays and pois_arrays on the caller's arrays equals
    the same step through the context API, bit for bit; the context's own
    arrays are untouched while the caller's are bound."""
    torch = pytest.importorskip("torch")
    cfg = getattr(config, name)
    init, coef = setup(cfg)
    ref = Box(cfg, init, coef)
    box = Box(cfg, init, coef)
    arr = _caller_arrays(torch, init)
    ptr = {n: arr[n].data_ptr() for n in FIELDS}
    for m in (1, 2, 3):
        ref.substep(m, m == 1)
        box.rhsp_arrays(ptr, m, m == 1)
        box.outflow_correction_arrays(ptr)
        box.pois_arrays(ptr, m)
    box.sync()
    _same(torch, ref, arr)
    # otbl_get_field reads the bound arrays
    for n in FIELDS:
        assert np.array_equal(box.field(n), ref.field(n)), n
    assert ref.inflow()[1]["dt"] == box.inflow()[1]["dt"]
    # back to the context's own arrays: still the initial state
    box.bind_state(None)
    for n in FIELDS:
        assert np.array_equal(box.field(n), np.asarray(init[n], dtype=np.float64).reshape(box.shape(n))), n
    # and re-bound: the context API continues on the caller's arrays
    box.bind_state(ptr)
    box.advance(1)
    ref.advance(1)
    box.sync()
    _same(torch, ref, arr)


def test_boun_and_genflu_on_caller_arrays():
    torch = pytest.importorskip("torch")
    cfg = config.SMALL
    init, coef = setup(cfg)
    ref = Box(cfg, init, coef)
    box = Box(cfg, init, coef)
    ref.substep(1, True)
    state = dict(init)
    state.update({n: ref.field(n) for n in FIELDS})
    arr = _caller_arrays(torch, state)
    ptr = {n: arr[n].data_ptr() for n in FIELDS}
    box.bind_state(ptr)
    box.sync()
    # genflu needs the same dt and clock: take the reference's inflow state
    um, st = ref.inflow()
    s = native.OtblInflow()
    for k, v in st.items():
        setattr(s, k, v)
    box.L.otbl_set_inflow(box.h, native.dptr(np.ascontiguousarray(init["u0"])),
                          native.dptr(np.ascontiguousarray(init["v0"])), native.dptr(um), ctypes.byref(s))
    ref.boun()
    box.boun_arrays(ptr)
    ref.genflu()
    box.genflu_arrays(ptr)
    box.sync()
    _same(torch, ref, arr)
    assert np.array_equal(box.inflow()[0], ref.inflow()[0])


def test_bind_refusals():
    torch = pytest.importorskip("torch")
    init, coef = setup(config.TINY)
    box = Box(config.TINY, init, coef)
    arr = _caller_arrays(torch, init)
    ptr = {n: arr[n].data_ptr() for n in FIELDS}
    L = box.L
    P = ctypes.c_void_p
    bad = [P(ptr[n]) for n in FIELDS]
    bad[0] = P(ptr["u"] + 8)  # not 16-byte aligned
    assert L.otbl_bind_state(box.h, *bad) == native.ERRORS_BY_NAME["ARG"]
    assert L.otbl_rhsp_arrays(box.h, *([None] * 7), 1, 1) == native.ERRORS_BY_NAME["ARG"]
    mixed = Box(replace(config.TINY, precision=1), init, coef)
    assert mixed.L.otbl_bind_state(mixed.h, *[P(ptr[n]) for n in FIELDS]) == native.ERRORS_BY_NAME["CONFIG"]
    # all NULL on the mixed path: its own arrays, nothing to refuse
    assert mixed.L.otbl_bind_state(mixed.h, *([None] * 7)) == 0
