"""Host-side mirror of the reference's substep interface.

``Box`` owns one device context (one boundary-layer box resident in HBM) and
exposes the reference's subroutine surface with the same meaning and order:

  rhsp(m, setstep)        rhsp.F90:22    RHS, RK3 stage update, implicit y
  outflow_correction()    boun.f90:63    global mass balance at the outflow
  pois(m)                 pois.f90:11    pressure Poisson solve + projection
  substep(m, setstep)     bl_1.F90:98-119 (the three calls above)
  advance(nsteps)         bl_1.F90:85-128 (3 substeps per step, tiempo += dt)
  boun(), genflu()        boun.f90:7, genflu.F90:3 (standalone pieces)
  chp2x/chx2p, fourxz, cosftx   change.f90, ffts.f90 on device buffers

State arrays use the reference's plane layout, as numpy arrays shaped
(nx, ny+1 or ny, nz1) -- C order of the Fortran (0:nz2, j, i) arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native
from .config import BoxConfig
from .native import FIELDS, UTYPE, OtblError, OtblInflow


class Box:
    def __init__(self, cfg: BoxConfig, init: dict, coef: np.ndarray | None = None,
                 device: int = 0):
        self.cfg = cfg
        self.L = native.lib()
        self.re = float(init["re"])
        self.xout = int(init["xout"])
        self.y = np.asarray(init["y"], dtype=np.float64)
        if coef is None:
            coef = native.coef_compute(cfg, self.re, self.xout, self.y, init["u0"])
        self.coef = np.ascontiguousarray(coef, dtype=np.float64)
        self.ccfg = native.make_config(cfg, self.re, self.xout)
        h = ctypes.c_void_p()
        st = self.L.otbl_ctx_create(ctypes.byref(self.ccfg), native.dptr(self.coef), device,
                                    ctypes.byref(h))
        self.h = h
        if st != native.OTBL_OK:
            msg = self.L.otbl_last_error(h).decode() if h.value else ""
            self.close()
            raise OtblError(f"otbl_ctx_create: {native.ERRORS.get(st, st)} {msg}")
        self.load(init)

    def rebind(self, cfg: BoxConfig, init: dict, coef: np.ndarray | None = None):
        """Re-use this context for another box of the same nx, ny, nz and
        precision (otbl_ctx_rebind), then upload its state."""
        re, xout = float(init["re"]), int(init["xout"])
        y = np.asarray(init["y"], dtype=np.float64)
        if coef is None:
            coef = native.coef_compute(cfg, re, xout, y, init["u0"])
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        ccfg = native.make_config(cfg, re, xout)
        self._check(self.L.otbl_ctx_rebind(self.h, ctypes.byref(ccfg), native.dptr(coef)),
                    "otbl_ctx_rebind")
        self.cfg, self.re, self.xout, self.y, self.coef, self.ccfg = cfg, re, xout, y, coef, ccfg
        self.load(init)

    def load(self, init: dict):
        """Upload a state: the seven fields and the genmod inflow state
        (getstartzy-bg.F90:18-297, :490-581)."""
        for n in FIELDS:
            self.set_field(n, init[n])
        inf = OtblInflow()
        inf.dt = float(init.get("dt", 0.0))
        inf.tiempo = float(init.get("tiempo", 0.0))
        inf.timeinit = float(init.get("timeinit", 0.0))
        self._check(self.L.otbl_set_inflow(
            self.h, native.dptr(np.ascontiguousarray(init["u0"], dtype=np.float64)),
            native.dptr(np.ascontiguousarray(init["v0"], dtype=np.float64)),
            native.dptr(np.ascontiguousarray(init["um"], dtype=np.float64)), ctypes.byref(inf)),
            "otbl_set_inflow")

    # ---- plumbing ----
    def _check(self, st, what):
        if st != native.OTBL_OK:
            msg = self.L.otbl_last_error(self.h).decode() if self.h else ""
            raise OtblError(f"{what}: {native.ERRORS.get(st, st)} {msg}")

    def shape(self, name):
        c = self.cfg
        return (c.nx, c.ny + 1 if UTYPE[name] else c.ny, c.nz1)

    def set_field(self, name, arr):
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64).reshape(self.shape(name)))
        self._check(self.L.otbl_set_field(self.h, FIELDS.index(name), native.dptr(a)), "otbl_set_field")

    def field(self, name) -> np.ndarray:
        a = np.empty(self.shape(name))
        self._check(self.L.otbl_get_field(self.h, FIELDS.index(name), native.dptr(a)), "otbl_get_field")
        return a

    def device_ptr(self, name) -> int:
        p = ctypes.POINTER(ctypes.c_double)()
        self._check(self.L.otbl_field_device_ptr(self.h, FIELDS.index(name), ctypes.byref(p)),
                    "otbl_field_device_ptr")
        return ctypes.cast(p, ctypes.c_void_p).value

    def inflow(self):
        um = np.zeros(self.cfg.ny + 1)
        st = OtblInflow()
        self._check(self.L.otbl_get_inflow(self.h, native.dptr(um), ctypes.byref(st)), "otbl_get_inflow")
        return um, {n: getattr(st, n) for n, _ in OtblInflow._fields_}

    def energies(self):
        """ener(1:15) as rhsp leaves it (rhsp.F90:116,487): energy integrals
        and wall-row values of plane nx/2 from the last substep m = 1."""
        e = np.zeros(15)
        self._check(self.L.otbl_get_energies(self.h, native.dptr(e)), "otbl_get_energies")
        return e

    @property
    def stream(self) -> int:
        """Raw cudaStream_t of the context (for torch.cuda.ExternalStream)."""
        h = ctypes.c_void_p()
        self._check(self.L.otbl_get_stream(self.h, ctypes.byref(h)), "otbl_get_stream")
        return h.value or 0

    def profile(self, on: bool):
        self._check(self.L.otbl_profile_enable(self.h, int(on)), "otbl_profile_enable")

    def profile_read(self) -> dict:
        """{kernel class: (total device ms, launches)} since profile(True)."""
        out = {}
        k = 0
        while True:
            name = ctypes.c_char_p()
            ms = ctypes.c_double()
            n = ctypes.c_int()
            if self.L.otbl_profile_read(self.h, k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(n)) != 0:
                break
            if n.value:
                out[name.value.decode()] = (ms.value, n.value)
            k += 1
        return out

    @property
    def launches(self) -> int:
        return int(self.L.otbl_launch_count(self.h))

    @property
    def device_bytes(self) -> int:
        return int(self.L.otbl_device_bytes(self.h))

    # ---- the reference's subroutine surface ----
    def rhsp(self, m: int, setstep: bool):
        self._check(self.L.otbl_rhsp(self.h, m, int(setstep)), "otbl_rhsp")

    def outflow_correction(self):
        self._check(self.L.otbl_outflow_correction(self.h), "otbl_outflow_correction")

    def pois(self, m: int):
        self._check(self.L.otbl_pois(self.h, m), "otbl_pois")

    def substep(self, m: int, setstep: bool):
        self._check(self.L.otbl_substep(self.h, m, int(setstep)), "otbl_substep")

    def advance(self, nsteps: int):
        self._check(self.L.otbl_advance(self.h, nsteps), "otbl_advance")

    def sync(self):
        self._check(self.L.otbl_sync(self.h), "otbl_sync")

    def autotune(self) -> tuple:
        """CTA sizes for k_interpx, k_difvisx, k_interpy picked by timing."""
        ch = (ctypes.c_int * 3)()
        self._check(self.L.otbl_autotune(self.h, ch), "otbl_autotune")
        return tuple(ch)

    def set_tuning(self, bs):
        ch = (ctypes.c_int * 3)(*bs)
        self._check(self.L.otbl_set_tuning(self.h, ch), "otbl_set_tuning")

    def busy(self) -> bool:
        """True while work issued on the context is in flight (never blocks)."""
        st = self.L.otbl_query(self.h)
        if st == native.OTBL_BUSY:
            return True
        self._check(st, "otbl_query")
        return False

    def boun(self):
        self._check(self.L.otbl_boun(self.h), "otbl_boun")

    def genflu(self):
        self._check(self.L.otbl_genflu(self.h), "otbl_genflu")

    NSTATS = 40

    def statsp(self):
        """One sample of the one-point statistics of the current state into
        the context's accumulators (statsp, stotf.F90:51-291)."""
        self._check(self.L.otbl_statsp(self.h), "otbl_statsp")

    def stats(self):
        """(accumulators (NSTATS, nx, ny) in the order of OTBL_ST_*, samples)."""
        out = np.zeros((self.NSTATS, self.cfg.nx, self.cfg.ny))
        n = ctypes.c_int()
        self._check(self.L.otbl_get_stats(self.h, native.dptr(out), ctypes.byref(n)), "otbl_get_stats")
        return out, n.value

    def reset_stats(self):
        self._check(self.L.otbl_reset_stats(self.h), "otbl_reset_stats")

    def interpyy(self):
        """lip.f90:359-440 on the state's u, w, v: (uy, wy, vy), ny rows each."""
        shp = (self.cfg.nx, self.cfg.ny, self.cfg.nz1)
        out = [np.zeros(shp) for _ in range(3)]
        self._check(self.L.otbl_interpyy(self.h, *[native.dptr(a) for a in out]), "otbl_interpyy")
        return tuple(out)

    # device-buffer pieces (pointers are raw device addresses)
    def chp2x(self, pen_dev: int, plan_dev: int, jee: int):
        """change.f90:224 chp2x(pen, plan, ...): planes -> pencils."""
        self._check(self.L.otbl_chp2x(self.h, pen_dev, plan_dev, jee), "otbl_chp2x")

    def chx2p(self, pen_dev: int, plan_dev: int, jee: int):
        """change.f90:257 chx2p(pen, plan, ...): pencils -> planes."""
        self._check(self.L.otbl_chx2p(self.h, pen_dev, plan_dev, jee), "otbl_chx2p")

    def fourxz(self, fou_dev: int, phys_dev: int, iopt: int, nlines: int):
        self._check(self.L.otbl_fourxz(self.h, fou_dev, phys_dev, iopt, nlines), "otbl_fourxz")

    def cosftx(self, c_dev: int, nlines: int, iopt: int):
        self._check(self.L.otbl_cosftx(self.h, c_dev, nlines, iopt), "otbl_cosftx")

    # ---- the reference's array surface (caller-owned device arrays, FP64) ----
    def _ptrs(self, arrays: dict, names):
        return [ctypes.c_void_p(int(arrays[n])) if arrays.get(n) else None for n in names]

    def bind_state(self, arrays: dict | None = None):
        """Points the state at caller-owned device arrays {field name: device
        address}; fields not given go back to the context's own arrays."""
        p = self._ptrs(arrays or {}, FIELDS)
        self._check(self.L.otbl_bind_state(self.h, *p), "otbl_bind_state")

    def rhsp_arrays(self, arrays: dict, m: int, setstep: bool):
        """rhsp(ut,vt,wt,pt,rhsupat,rhsvpat,rhswpat,...), rhsp.F90:22-27."""
        self._check(self.L.otbl_rhsp_arrays(self.h, *self._ptrs(arrays, FIELDS), m, int(setstep)),
                    "otbl_rhsp_arrays")

    def outflow_correction_arrays(self, arrays: dict):
        """outflow_correction(ut,vt,rhsupat,...), boun.f90:63."""
        self._check(self.L.otbl_outflow_correction_arrays(
            self.h, *self._ptrs(arrays, ("u", "v", "rhsupa"))), "otbl_outflow_correction_arrays")

    def pois_arrays(self, arrays: dict, m: int):
        """pois(ut,vt,wt,pt,res,rest,rt,varstep,...), pois.f90:11."""
        self._check(self.L.otbl_pois_arrays(self.h, *self._ptrs(arrays, ("u", "v", "w", "p")), m),
                    "otbl_pois_arrays")

    def boun_arrays(self, arrays: dict):
        """boun(ut,vt,wt), boun.f90:7."""
        self._check(self.L.otbl_boun_arrays(self.h, *self._ptrs(arrays, ("u", "v", "w"))),
                    "otbl_boun_arrays")

    def genflu_arrays(self, arrays: dict):
        """genflu(ut,vt,wt,...), genflu.F90:3."""
        self._check(self.L.otbl_genflu_arrays(self.h, *self._ptrs(arrays, ("u", "v", "w"))),
                    "otbl_genflu_arrays")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.otbl_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_box(cfg: BoxConfig, device: int = 0):
    """Seeded synthetic box (opentbl_b200.synth) resident on the device."""
    from . import synth
    init = synth.make_initial(cfg)
    return Box(cfg, init, device=device), init
