"""ORACLE (test infrastructure only): ctypes binding of oracle/liboracle.so.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline, as the checker / the timed CPU port of the reference's substep.
Parity of this restatement with the reference is UNPINNED (no reference
tests or golden outputs exist, and the Fortran cannot be built here).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


class OtblConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xout", ctypes.c_int), ("xpose_round", ctypes.c_int),
                ("dt_mode", ctypes.c_int), ("re", ctypes.c_double),
                ("ax", ctypes.c_double), ("ay", ctypes.c_double),
                ("az", ctypes.c_double), ("cfl", ctypes.c_double),
                ("y_blend", ctypes.c_double), ("dt_fixed", ctypes.c_double),
                ("precision", ctypes.c_int), ("options", ctypes.c_int)]


class OtblInflow(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("tiempo", "timeinit", "dt", "utauout", "rthout", "dout",
                 "gamma1", "gamma2", "timec", "umax", "wmax", "vmax")]


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.orc_coef_compute.argtypes = [ctypes.POINTER(OtblConfig), D, D, D]
        L.orc_coef_compute.restype = ctypes.c_int
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(OtblConfig), D]
        L.orc_destroy.argtypes = [P]
        L.orc_field.restype = D
        L.orc_field.argtypes = [P, ctypes.c_int]
        L.orc_set_inflow.argtypes = [P, D, D, D, ctypes.POINTER(OtblInflow)]
        L.orc_get_inflow.argtypes = [P, D, ctypes.POINTER(OtblInflow)]
        L.orc_get_energies.argtypes = [P, D]
        for n in ("orc_rhsp", "orc_substep"):
            getattr(L, n).argtypes = [P, ctypes.c_int, ctypes.c_int]
            getattr(L, n).restype = ctypes.c_int
        L.orc_advance.argtypes = [P, ctypes.c_int]
        L.orc_advance.restype = ctypes.c_int
        L.orc_pois.argtypes = [P, ctypes.c_int]
        for n in ("orc_outflow_correction", "orc_boun", "orc_genflu"):
            getattr(L, n).argtypes = [P]
        L.orc_divergence.argtypes = [P, D]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_interpxx.argtypes = [P, D, D, ctypes.c_int, ctypes.c_int]
        L.orc_difvisxx.argtypes = [P, D, D, D, ctypes.c_int, ctypes.c_int]
        L.orc_interpyy.argtypes = [P, D, D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_differzy.argtypes = [P, D, D, ctypes.c_int]
        L.orc_vistyy.argtypes = [P, D, D, ctypes.c_int]
        L.orc_implzy.argtypes = [P, D, D, ctypes.c_int, ctypes.c_double]
        L.orc_fourxz.argtypes = [P, D, D, ctypes.c_int, ctypes.c_int]
        L.orc_cosftx.argtypes = [P, D, ctypes.c_int, ctypes.c_int]
        L.orc_chp2x.argtypes = [P, D, D, ctypes.c_int]
        L.orc_chx2p.argtypes = [P, D, D, ctypes.c_int]
        L.orc_fft_create.restype = P
        L.orc_fft_create.argtypes = [ctypes.c_int]
        L.orc_fft_destroy.argtypes = [P]
        L.orc_fft_exec.argtypes = [P, D, D, ctypes.c_int]
        L.orc_c2r_line.argtypes = [P, ctypes.c_int, ctypes.c_int, D, D, D]
        L.orc_r2c_line.argtypes = [P, ctypes.c_int, ctypes.c_int, D, D, D]
        L.orc_dct_line.argtypes = [P, ctypes.c_int, D, ctypes.c_int, D]
        L.orc_statsp.argtypes = [P, D]
        L.orc_stats_operator.argtypes = [P, ctypes.c_int, D, D]
        _lib = L
    return _lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


FIELDS = ("u", "v", "w", "p", "rhsupa", "rhsvpa", "rhswpa")
UTYPE = {"u": True, "v": False, "w": True, "p": False,
         "rhsupa": True, "rhsvpa": False, "rhswpa": True}


def make_config(cfg, re: float, xout: int) -> OtblConfig:
    return OtblConfig(cfg.nx, cfg.ny, cfg.nz, xout, cfg.xpose_round, cfg.dt_mode,
                      re, cfg.ax, 0.0, cfg.az, cfg.cfl, cfg.y_blend, cfg.dt_fixed,
                      getattr(cfg, "precision", 0), getattr(cfg, "options", 0))


def coef_count(cfg) -> int:
    """Length of the packed coefficient buffer (include/otbl_layout.h)."""
    nx, ny, nz2 = cfg.nx, cfg.ny, cfg.nz2
    lens = [64, ny + 2, ny + 1, ny + 1, ny, ny, ny + 1, nx + 2, nx + 1, nz2 + 1, nz2 + 1,
            nz2 + 1, nx - 1, 3 * ny, nx, 3 * nx, 3 * nx, 2 * nx, 2 * nx, 16, 3 * nx, 3 * nx,
            2 * nx, 2 * nx, 20, 3 * nx, 3 * nx, 3 * nx, 3 * nx, 16, 3 * ny, 3 * ny, 2 * ny,
            2 * ny, 16, 3 * (ny + 1), 3 * ny, 2 * ny, 2 * ny, 16, 3 * (ny + 1), 3 * ny,
            3 * (ny + 1), 3 * ny, 3 * ny, 3 * ny, 16, 8,
            8 * ny, 8 * nx, 8 * nx, 8 * ny, 8 * ny]
    return int(sum(lens))


def coef_compute(cfg, re: float, xout: int, y: np.ndarray, u0: np.ndarray) -> np.ndarray:
    """The oracle's own coefficient set-up (oracle/orc_coef.c: coeft.f90
    coef, bl_1.F90 wavenumbers and inlet_retheta, boun.f90 magicnumber)."""
    L = lib()
    c = make_config(cfg, re, xout)
    out = np.zeros(coef_count(cfg))
    st = L.orc_coef_compute(ctypes.byref(c), dptr(np.ascontiguousarray(y, dtype=np.float64)),
                            dptr(np.ascontiguousarray(u0, dtype=np.float64)), dptr(out))
    if st != 0:
        raise RuntimeError(f"orc_coef_compute failed: {st}")
    return out


class OracleBox:
    """CPU restatement of one box; same state layout as the product. Its
    coefficients come from the oracle's own set-up (coef_compute) on the
    box's grid y, inlet profile u0, Re and xout."""

    def __init__(self, cfg, init: dict, threads: int = 0):
        self.cfg = cfg
        self.L = lib()
        if threads:
            self.L.orc_set_threads(threads)
        self.ccfg = make_config(cfg, init["re"], init["xout"])
        self.coef = coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
        self.h = self.L.orc_create(ctypes.byref(self.ccfg), dptr(self.coef))
        for i, n in enumerate(FIELDS):
            self.set_field(n, init[n])
        st = OtblInflow()
        st.dt = init.get("dt", 0.0)
        st.tiempo = init.get("tiempo", 0.0)
        st.timeinit = init.get("timeinit", 0.0)
        self.L.orc_set_inflow(self.h, dptr(np.ascontiguousarray(init["u0"])),
                              dptr(np.ascontiguousarray(init["v0"])),
                              dptr(np.ascontiguousarray(init["um"])), ctypes.byref(st))

    def _shape(self, name):
        c = self.cfg
        return (c.nx, c.ny + 1 if UTYPE[name] else c.ny, c.nz1)

    def field_view(self, name):
        ptr = self.L.orc_field(self.h, FIELDS.index(name))
        n = int(np.prod(self._shape(name)))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self._shape(name))

    def field(self, name):
        return self.field_view(name).copy()

    def set_field(self, name, arr):
        self.field_view(name)[...] = np.asarray(arr, dtype=np.float64).reshape(self._shape(name))

    def inflow(self):
        um = np.zeros(self.cfg.ny + 1)
        st = OtblInflow()
        self.L.orc_get_inflow(self.h, dptr(um), ctypes.byref(st))
        return um, {n: getattr(st, n) for n, _ in OtblInflow._fields_}

    def energies(self):
        e = np.zeros(15)
        self.L.orc_get_energies(self.h, dptr(e))
        return e

    def rhsp(self, m, setstep):
        return self.L.orc_rhsp(self.h, m, setstep)

    def outflow_correction(self):
        self.L.orc_outflow_correction(self.h)

    def pois(self, m):
        self.L.orc_pois(self.h, m)

    def substep(self, m, setstep):
        return self.L.orc_substep(self.h, m, setstep)

    def advance(self, nsteps):
        st = self.L.orc_advance(self.h, nsteps)
        if st != 0:
            raise RuntimeError(f"oracle advance failed: {st}")

    NSTATS = 40

    def statsp(self, acc: np.ndarray | None = None) -> np.ndarray:
        """Adds one sample of statsp (stotf.F90:51-291) of the current state
        to acc, (NSTATS, nx, ny) (the reference's (ny, nx) per statistic),
        and returns it."""
        c = self.cfg
        if acc is None:
            acc = np.zeros((self.NSTATS, c.nx, c.ny))
        self.L.orc_statsp(self.h, dptr(acc))
        return acc

    def stats_operator(self, op: int, line: np.ndarray, n_out: int) -> np.ndarray:
        """One line/column through a statistics operator: 0 interpx_new, 1
        diffx, 2 interpy_new (u), 3 interpy_new (p), 4 diffy."""
        out = np.zeros(n_out)
        self.L.orc_stats_operator(self.h, op, dptr(np.ascontiguousarray(line, dtype=np.float64)), dptr(out))
        return out

    def divergence(self):
        c = self.cfg
        d = np.zeros((c.nx, c.ny, c.nz1))
        self.L.orc_divergence(self.h, dptr(d))
        return d

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
