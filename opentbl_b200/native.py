"""ctypes binding of the in-tree CUDA library opentbl_b200/libotbl.so.

The library is the product: every substep kernel runs there. There is no
CPU fallback -- if the library is missing or no CUDA device is usable, the
calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libotbl.so")
_lib = None

OTBL_OK = 0
OTBL_BUSY = 7
ERRORS = {1: "bad argument", 2: "bad configuration", 3: "out of device memory",
          4: "CUDA error", 5: "non-finite value", 6: "no CUDA device",
          8: "device wait timed out"}
ERRORS_BY_NAME = {"ARG": 1, "CONFIG": 2, "OOM": 3, "CUDA": 4, "NAN": 5, "NODEV": 6, "BUSY": 7,
                  "TIMEOUT": 8}
FIELDS = ("u", "v", "w", "p", "rhsupa", "rhsvpa", "rhswpa")
UTYPE = {"u": True, "v": False, "w": True, "p": False,
         "rhsupa": True, "rhsvpa": False, "rhswpa": True}

# order of include/otbl_layout.h OTBL_COEF_LIST
COEF_NAMES = ("SCAL", "Y", "DY", "IDY", "IDYY", "DYMIN", "HY", "XG", "DX", "KAZ",
              "KAZ2", "KVIS", "KMOD", "AYP", "VMAGIC", "INXU", "INXV", "COFIUX",
              "COFIVX", "INBX", "DCXU", "DCXV", "COFCXU", "COFCXV", "DCBX", "VIXU",
              "VIXV", "COFVXU", "COFVXV", "COFVBX", "INYU", "INYV", "COFIUY",
              "COFIVY", "INBY", "DCYU", "DCYV", "COFCYU", "COFCYV", "DCBY", "VIYU",
              "VIYV", "VYUI", "VYVI", "COFVYU", "COFVYV", "COFVBY", "CCON",
              "FD_DVDY", "FD_DX", "FD_IX", "FD_IY", "FD_IYP")
SCAL = dict(RE=0, REX=1, AX=2, AY=3, AZ=4, CFL=5, DX1=6, IDX=7, IDXX=8, DXMIN=9,
            DZMIN=10, DTRET=11, PI=12, UINF=13, RTHIN=14, DIN=15, YBLEND=16,
            RKC=20, RKD=23, RKCV=26, RKDV=29, NX=40, NY=41, NZ=42, XOUT=43)


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


class OtblError(RuntimeError):
    pass


def _bind(L):
    P = ctypes.c_void_p
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.c_int
    sig = {
        "otbl_config_check": ([ctypes.POINTER(OtblConfig)], I),
        "otbl_coef_count": ([I, I, I], ctypes.c_size_t),
        "otbl_coef_offset": ([I, I, I, I, ctypes.POINTER(ctypes.c_size_t)], I),
        "otbl_coef_compute": ([ctypes.POINTER(OtblConfig), D, D, D], I),
        "otbl_ctx_create": ([ctypes.POINTER(OtblConfig), D, I, ctypes.POINTER(P)], I),
        "otbl_ctx_destroy": ([P], None),
        "otbl_last_error": ([P], ctypes.c_char_p),
        "otbl_device_bytes": ([P], ctypes.c_size_t),
        "otbl_ctx_bytes": ([ctypes.POINTER(OtblConfig)], ctypes.c_size_t),
        "otbl_ctx_rebind": ([P, ctypes.POINTER(OtblConfig), D], I),
        "otbl_set_field": ([P, I, D], I),
        "otbl_get_field": ([P, I, D], I),
        "otbl_field_device_ptr": ([P, I, ctypes.POINTER(D)], I),
        "otbl_set_inflow": ([P, D, D, D, ctypes.POINTER(OtblInflow)], I),
        "otbl_get_inflow": ([P, D, ctypes.POINTER(OtblInflow)], I),
        "otbl_get_energies": ([P, D], I),
        "otbl_rhsp": ([P, I, I], I),
        "otbl_outflow_correction": ([P], I),
        "otbl_pois": ([P, I], I),
        "otbl_substep": ([P, I, I], I),
        "otbl_advance": ([P, I], I),
        "otbl_sync": ([P], I),
        "otbl_chp2x": ([P, P, P, I], I),
        "otbl_chx2p": ([P, P, P, I], I),
        "otbl_fourxz": ([P, P, P, I, I], I),
        "otbl_cosftx": ([P, P, I, I], I),
        "otbl_boun": ([P], I),
        "otbl_interpyy": ([P, D, D, D], I),
        "otbl_genflu": ([P], I),
        "otbl_statsp": ([P], I),
        "otbl_get_stats": ([P, D, ctypes.POINTER(I)], I),
        "otbl_reset_stats": ([P], I),
        "otbl_bind_state": ([P] + [P] * 7, I),
        "otbl_rhsp_arrays": ([P] + [P] * 7 + [I, I], I),
        "otbl_outflow_correction_arrays": ([P, P, P, P], I),
        "otbl_pois_arrays": ([P, P, P, P, P, I], I),
        "otbl_boun_arrays": ([P, P, P, P], I),
        "otbl_genflu_arrays": ([P, P, P, P], I),
        "otbl_launch_count": ([P], ctypes.c_longlong),
        "otbl_graph_create": ([ctypes.POINTER(P), I, I, ctypes.POINTER(P)], I),
        "otbl_graph_launch": ([P], I),
        "otbl_graph_sync": ([P], I),
        "otbl_graph_query": ([P], I),
        "otbl_graph_stream": ([P, ctypes.POINTER(P)], I),
        "otbl_graph_kernels": ([P], ctypes.c_longlong),
        "otbl_graph_destroy": ([P], None),
        "otbl_query": ([P], I),
        "otbl_autotune": ([P, ctypes.POINTER(ctypes.c_int)], I),
        "otbl_set_tuning": ([P, ctypes.POINTER(ctypes.c_int)], I),
        "otbl_selftest_wait": ([P, ctypes.POINTER(ctypes.c_int)], I),
        "otbl_get_stream": ([P, ctypes.POINTER(P)], I),
        "otbl_profile_enable": ([P, I], I),
        "otbl_profile_read": ([P, I, ctypes.POINTER(ctypes.c_char_p), D, ctypes.POINTER(I)], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


def lib():
    """Loads libotbl.so (building it first if sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        _lib = _bind(ctypes.CDLL(LIB_PATH))
    return _lib


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_config(cfg, re: float, xout: int) -> OtblConfig:
    return OtblConfig(cfg.nx, cfg.ny, cfg.nz, xout, cfg.xpose_round, cfg.dt_mode,
                      re, cfg.ax, 0.0, cfg.az, cfg.cfl, cfg.y_blend, cfg.dt_fixed,
                      getattr(cfg, "precision", 0), getattr(cfg, "options", 0))


def coef_compute(cfg, re: float, xout: int, y: np.ndarray, u0: np.ndarray) -> np.ndarray:
    """Packed coefficient buffer (coeft.f90 coef + inlet_retheta + magicnumber)."""
    L = lib()
    c = make_config(cfg, re, xout)
    n = L.otbl_coef_count(cfg.nx, cfg.ny, cfg.nz)
    out = np.zeros(n)
    st = L.otbl_coef_compute(ctypes.byref(c), dptr(np.ascontiguousarray(y, dtype=np.float64)),
                             dptr(np.ascontiguousarray(u0, dtype=np.float64)), dptr(out))
    if st != OTBL_OK:
        raise OtblError(f"otbl_coef_compute: {ERRORS.get(st, st)}")
    return out


def coef_offsets(cfg) -> dict:
    L = lib()
    res = {}
    for i, name in enumerate(COEF_NAMES + ("TOTAL",)):
        off = ctypes.c_size_t()
        L.otbl_coef_offset(cfg.nx, cfg.ny, cfg.nz, i, ctypes.byref(off))
        res[name] = off.value
    return res
