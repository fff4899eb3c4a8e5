"""Ensembles of independent boxes advanced together (no counterpart in the
reference, which runs one box per MPI job).

`Graph` wraps otbl_graph_*: the RK3 steps of many contexts captured into one
CUDA graph whose branches run concurrently, so one launch advances the whole
ensemble. `ensemble_configs` draws the boxes of a parameter sweep in inlet
Re_theta and domain size from a seed.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native
from .config import BoxConfig


class Graph:
    """nsteps RK3 steps of every box in `boxes` (Box objects on one device)
    as one CUDA graph. Destroy it (close) before the boxes."""

    def __init__(self, boxes, nsteps: int):
        self.L = native.lib()
        self.boxes = list(boxes)
        self.nsteps = nsteps
        arr = (ctypes.c_void_p * len(self.boxes))(*[b.h.value for b in self.boxes])
        h = ctypes.c_void_p()
        st = self.L.otbl_graph_create(arr, len(self.boxes), nsteps, ctypes.byref(h))
        if st != native.OTBL_OK:
            raise native.OtblError(f"otbl_graph_create: {native.ERRORS.get(st, st)}")
        self.h = h

    @property
    def kernels(self) -> int:
        """Kernel launches per graph launch (all boxes)."""
        return int(self.L.otbl_graph_kernels(self.h))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self.L.otbl_graph_stream(self.h, ctypes.byref(s))
        return s.value or 0

    def launch(self):
        st = self.L.otbl_graph_launch(self.h)
        if st != native.OTBL_OK:
            raise native.OtblError(f"otbl_graph_launch: {native.ERRORS.get(st, st)}")

    def busy(self) -> bool:
        st = self.L.otbl_graph_query(self.h)
        if st == native.OTBL_BUSY:
            return True
        if st != native.OTBL_OK:
            raise native.OtblError(f"otbl_graph_query: {native.ERRORS.get(st, st)}")
        return False

    def sync(self):
        st = self.L.otbl_graph_sync(self.h)
        if st != native.OTBL_OK:
            raise native.OtblError(f"otbl_graph_sync: {native.ERRORS.get(st, st)}")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.otbl_graph_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NX = (129, 257, 385, 513)
NY = (65, 97, 129)
NZ = (64, 128, 256)


def ensemble_configs(n: int = 24, seed: int = 2024, precision: int = 1) -> list[BoxConfig]:
    """n boxes of a seeded sweep: nx in {129, 257, 385, 513}, ny in {65, 97,
    129}, nz in {64, 128, 256}, inlet Re_theta ~ U[300, 1500], Lx ~ U[40, 80],
    Lz ~ U[6, 10] (delta0 units), Ly = 8 with dy_wall = 0.002 as the
    257x97x128 box; Blasius inlet profile below Re_theta 700, Musker above;
    each box's perturbation seeded from the sweep seed."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx, ny, nz = int(rng.choice(NX)), int(rng.choice(NY)), int(rng.choice(NZ))
        rt = float(rng.uniform(300.0, 1500.0))
        lx = float(rng.uniform(40.0, 80.0))
        lz = float(rng.uniform(6.0, 10.0))
        out.append(BoxConfig(nx=nx, ny=ny, nz=nz, lx=lx, ly=8.0, lz=lz, dy_wall=0.002,
                             re_theta=rt, profile="blasius" if rt < 700.0 else "musker",
                             precision=precision, seed=int(rng.integers(1, 2**31 - 1)),
                             name=f"ens{k:02d}-{nx}x{ny}x{nz}"))
    return out
