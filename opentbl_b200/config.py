"""Box configurations (the reference's input deck, bl_1.F90:203-230, plus the
compile-time sizes of mod.F90:22-23, which are runtime values here).

Lengths are in units of the inlet boundary-layer thickness delta0 = 1 and
velocities in units of U_inf = 1. The reference's streamwise coordinate is
x(i) = i*ax*pi/(nx+1) (coeft.f90:401-405), so Lx ~= ax*pi, and the spanwise
wavenumbers are k/az (bl_1.F90:360), so Lz = 2*pi*az.
"""
from __future__ import annotations

import dataclasses
import math


@dataclasses.dataclass
class BoxConfig:
    nx: int
    ny: int
    nz: int
    lx: float = 60.0
    ly: float = 8.0
    lz: float = 8.0
    dy_wall: float = 0.002
    re_theta: float = 300.0
    profile: str = "blasius"          # "blasius" | "musker"
    cfl: float = 0.5
    xout: int = 0                      # 0: chosen by default_xout()
    y_blend: float = 1.5               # replaces y(119) in genflu.F90:57
    xpose_round: int = 0               # 0 none, 1 fp32 (REAL4 transposes)
    dt_mode: int = 0                   # 0 adaptive (reference), 1 fixed
    dt_fixed: float = 0.0
    precision: int = 0                 # 0 FP64, 1 mixed (OTBL_PREC_*)
    options: int = 0                   # OTBL_OPT_* bits (1: interpyy on the tensor cores)
    amp: float = 0.05                  # perturbation amplitude / U_inf
    seed: int = 1234
    name: str = ""

    @property
    def nz1(self) -> int:
        return 2 * (self.nz // 3)

    @property
    def nz2(self) -> int:
        return self.nz1 // 2 - 1

    @property
    def ax(self) -> float:
        return self.lx / math.pi

    @property
    def az(self) -> float:
        return self.lz / (2.0 * math.pi)

    def default_xout(self) -> int:
        """Recycling plane about 10 delta0 downstream of the inlet (the
        reference hard-codes xout=600 of nx=4097, mod.F90:23)."""
        dx = self.lx / (self.nx + 1)
        return int(min(max(5, 1 + round(10.0 / dx)), self.nx // 2))

    def resolved_xout(self) -> int:
        return self.xout if self.xout > 0 else self.default_xout()

    @property
    def mpts(self) -> float:
        """Grid points in millions, the unit of the headline metric."""
        return self.nx * self.ny * self.nz / 1e6


# 257x97x128, Re_theta=300, Lx=60, Ly=8 (dy_wall=0.002), Lz=8
C1 = BoxConfig(nx=257, ny=97, nz=128, lx=60.0, ly=8.0, lz=8.0, re_theta=300.0,
               profile="blasius", name="C1-257x97x128")
# 1025x193x512, Re_theta=1000, Lx=80, Ly=10, Lz=10
C2 = BoxConfig(nx=1025, ny=193, nz=512, lx=80.0, ly=10.0, lz=10.0,
               re_theta=1000.0, profile="musker", name="C2-1025x193x512")
# medium box for profiling captures: fields of 135 MB (larger than L2),
# about 3.5 GB on the device
MED = BoxConfig(nx=513, ny=193, nz=256, lx=40.0, ly=10.0, lz=8.0,
                re_theta=1000.0, profile="musker", name="MED-513x193x256")
# a quarter of the 1025x193x512 box in x, same y and z sizes (every kernel
# takes the code path of the full box): fields of 135 MB, about 3.5 GB on the
# device, for profiling captures
SLAB = BoxConfig(nx=257, ny=193, nz=512, lx=20.0, ly=10.0, lz=10.0,
                 re_theta=1000.0, profile="musker", name="SLAB-257x193x512")
# the x extent of the 1025x193x512 box with a quarter of its rows (the x-line
# and x-DCT kernels take the code path of the full box, n = 1024): fields of
# 139 MB, about 3.6 GB on the device, for profiling captures
STRIP = BoxConfig(nx=1025, ny=49, nz=512, lx=80.0, ly=10.0, lz=10.0,
                  re_theta=1000.0, profile="musker", name="STRIP-1025x49x512")
# small box for tests and smoke runs
TINY = BoxConfig(nx=33, ny=41, nz=32, lx=12.0, ly=6.0, lz=4.0, dy_wall=0.02,
                 re_theta=300.0, profile="blasius", y_blend=1.5,
                 name="tiny-33x41x32")
SMALL = BoxConfig(nx=65, ny=57, nz=64, lx=24.0, ly=8.0, lz=6.0,
                  dy_wall=0.006, re_theta=300.0, profile="blasius",
                  name="small-65x57x64")


def replace(cfg: BoxConfig, **kw) -> BoxConfig:
    return dataclasses.replace(cfg, **kw)
