"""Seeded synthetic initial fields.

The reference always restarts from HDF5 files (getstartzy-bg.F90:18-297) and
has no field generator, so the initial condition is built here:

* y grid y(0:ny+1): tanh stretching with y(1) = 0 at the wall, y(ny) = Ly and
  first spacing dy_wall; y(0) and y(ny+1) mirror the first/last spacing.
* mean flow: a Blasius profile (laminar-like boxes) or a Musker inner law with
  a Coles wake (turbulent-like boxes), growing with x, with the mean V
  obtained from the discrete continuity equation of pois.f90:41-54 so the
  mean field is divergence-free row by row.
* perturbation of amplitude ``amp`` (peak |u'| / U_inf) from two seeded
  potentials whose discrete curls are divergence-free for the same stencil:
  psi(x,y) per spanwise mode for (u', v') and phi(y) per mode for (v', w').
  The spectrum peaks at kz*delta0 = 2 and is confined to y < 1.2 delta0.
* fields are rounded to FP32-representable values, as the reference's REAL4
  restart read does (getstartzy-bg.F90:98,110,128).

Everything is numpy and deterministic for a given BoxConfig (PCG64 seed).
"""
from __future__ import annotations

import math

import numpy as np

from .config import BoxConfig


def y_grid(cfg: BoxConfig) -> np.ndarray:
    """y(0:ny+1): wall at y(1)=0, top at y(ny)=Ly, y(2)-y(1) = dy_wall."""
    ny, ly, d1 = cfg.ny, cfg.ly, cfg.dy_wall
    s = np.arange(ny, dtype=np.float64) / (ny - 1)

    def grid(g):
        return ly * (1.0 - np.tanh(g * (1.0 - s)) / np.tanh(g))

    lo, hi = 1e-6, 20.0
    if grid(hi)[1] > d1 or ly / (ny - 1) < d1:
        raise ValueError("dy_wall not reachable with this ny/Ly")
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if grid(mid)[1] > d1:
            lo = mid
        else:
            hi = mid
    yy = grid(0.5 * (lo + hi))
    yy[0] = 0.0
    yy[-1] = ly
    y = np.empty(ny + 2)
    y[1:ny + 1] = yy
    y[0] = -(yy[1] - yy[0])
    y[ny + 1] = yy[-1] + (yy[-1] - yy[-2])
    return y


def _blasius_table():
    """f, f' of f''' + f f''/2 = 0, f(0)=f'(0)=0, f''(0)=0.332057336215."""
    h = 1e-3
    n = 12000
    z = np.array([0.0, 0.0, 0.332057336215196])
    eta = np.arange(n + 1) * h
    f = np.empty(n + 1)
    fp = np.empty(n + 1)

    def rhs(z):
        return np.array([z[1], z[2], -0.5 * z[0] * z[2]])

    for i in range(n + 1):
        f[i], fp[i] = z[0], z[1]
        k1 = rhs(z)
        k2 = rhs(z + 0.5 * h * k1)
        k3 = rhs(z + 0.5 * h * k2)
        k4 = rhs(z + h * k3)
        z = z + h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
    return eta, f, fp


_BLASIUS = None


def blasius(eta):
    global _BLASIUS
    if _BLASIUS is None:
        _BLASIUS = _blasius_table()
    e, f, fp = _BLASIUS
    eta = np.asarray(eta, dtype=np.float64)
    em = e[-1]
    fpv = np.interp(np.clip(eta, 0.0, em), e, fp)
    fv = np.interp(np.clip(eta, 0.0, em), e, f) + np.maximum(eta - em, 0.0)
    return fv, fpv


def _musker_table(ymax: float):
    """u+(y+) of Musker (1979): du+/dy+ = (y+^2/k + 1/s)/(y+^3 + y+^2/k + 1/s)."""
    kap, s = 0.41, 0.001093
    yp = np.concatenate([[0.0], np.geomspace(1e-3, max(ymax, 10.0), 4000)])
    g = (yp ** 2 / kap + 1.0 / s) / (yp ** 3 + yp ** 2 / kap + 1.0 / s)
    up = np.concatenate([[0.0], np.cumsum(0.5 * (g[1:] + g[:-1]) * np.diff(yp))])
    return yp, up


def _musker_profile(y, delta, re):
    """U(y)/U_inf for a boundary layer of thickness delta at Reynolds re."""
    kap, pi_w = 0.41, 0.45
    yp_t, up_t = _musker_table(re * delta * 0.2 + 100.0)
    utau = 0.04
    for _ in range(60):   # 1/utau = u+(delta+) + 2 Pi / kappa
        dplus = delta * utau * re
        utau = 1.0 / (np.interp(dplus, yp_t, up_t) + 2.0 * pi_w / kap)
    eta = np.clip(np.asarray(y) / delta, 0.0, None)
    yplus = np.clip(np.asarray(y), 0.0, None) * utau * re
    uplus = np.interp(yplus, yp_t, up_t) + (2.0 * pi_w / kap) * np.sin(0.5 * np.pi * np.minimum(eta, 1.0)) ** 2
    u = np.minimum(uplus * utau, 1.0)
    u[eta >= 1.0] = 1.0
    return u


def _theta_discrete(u0, y, re=1.0):
    """Re_theta / re of inlet_retheta (bl_1.F90:381-388)."""
    ny = len(y) - 2
    dy = np.diff(y)  # dy(0:ny)
    uinf = u0[ny + 1 - 20 - 1:ny + 1 - 5].sum() / 16.0
    u99 = float(np.float32(0.99)) * uinf
    jtop = 0
    for j in range(1, ny - 1):
        if u0[j - 1] >= u99:
            break
        jtop = j + 1
    uu = u0[1:jtop + 3]
    return float(((uinf - uu) * uu * dy[1:jtop + 3]).sum() / uinf)


def mean_profile(cfg: BoxConfig, y, delta, re):
    """U at the u/w rows yp(j) = (y(j-1)+y(j))/2, j=1..ny+1 (coeft.f90:234)."""
    yp = 0.5 * (y[:-1] + y[1:])
    if cfg.profile == "blasius":
        _, fp = blasius(4.91 * yp / delta)
        u = fp.copy()
    else:
        u = _musker_profile(yp, delta, re)
    u[0] = -u[1]    # ghost row below the wall, refreshed by boun anyway
    return u


def reynolds_for(cfg: BoxConfig, y) -> float:
    """Re such that inlet_retheta of the inlet profile gives cfg.re_theta."""
    if cfg.profile == "blasius":
        u0 = mean_profile(cfg, y, 1.0, 1.0)
        return cfg.re_theta / _theta_discrete(u0, y)
    lo, hi = 100.0, 1e7
    for _ in range(100):
        mid = math.sqrt(lo * hi)
        rt = mid * _theta_discrete(mean_profile(cfg, y, 1.0, mid), y)
        if rt < cfg.re_theta:
            lo = mid
        else:
            hi = mid
    return math.sqrt(lo * hi)


def _delta_of_x(cfg: BoxConfig, x, re):
    if cfg.profile == "blasius":
        x0 = re / 4.91 ** 2
        return np.sqrt((x + x0) / x0)
    # turbulent growth delta ~ x^0.8 with d(delta)/dx = 0.16 Re_x^-1/7 at x=0
    d0 = 1.0
    slope = 0.16 * (re * d0 / 0.37) ** (-1.0 / 7.0) * 0.8
    x0 = 0.8 * d0 / slope
    return d0 * ((x + x0) / x0) ** 0.8


def make_initial(cfg: BoxConfig) -> dict:
    """Returns the state of a fresh box in the reference layout:
    u, w: (nx, ny+1, nz1) ; v, p: (nx, ny, nz1) float64 (C order = the
    Fortran (0:nz2, j, i) order), plus y, re, u0, v0, um and xout."""
    nx, ny, nz1, nz2 = cfg.nx, cfg.ny, cfg.nz1, cfg.nz2
    y = y_grid(cfg)
    re = reynolds_for(cfg, y)
    dx = cfg.ax * math.pi / (nx + 1)
    x = np.arange(1, nx + 1) * dx - dx          # plane i at x(i) - x(1)
    delta = _delta_of_x(cfg, x, re)
    U = np.stack([mean_profile(cfg, y, d, re) for d in delta])   # (nx, ny+1)
    dy = np.diff(y)                              # dy(0:ny)
    # mean V from the discrete continuity of pois.f90:41-54 (k = 0, no w)
    V = np.zeros((nx, ny))
    for i in range(1, nx):
        dudx = (U[i, 1:ny] - U[i - 1, 1:ny]) / dx   # rows j+1 = 2..ny
        V[i, 1:] = -np.cumsum(dy[1:ny] * dudx)
    V[0] = V[1]

    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    kz = np.arange(nz2 + 1) / cfg.az
    spec = np.exp(-0.5 * ((kz - 2.0) / 1.0) ** 2)
    spec[0] = 0.0
    ywin = 1.2
    yv = y[1:ny + 1]                              # v rows y(1:ny)

    def window(yy):
        t = np.clip(yy / ywin, 0.0, 1.0)
        return (t * (1.0 - t)) ** 2 * 16.0

    # smooth random functions of x: a few Fourier components per mode
    nmod = 4
    lam = rng.uniform(3.0, 8.0, size=(2, nz2 + 1, nmod))
    ph = rng.uniform(0.0, 2 * np.pi, size=(2, nz2 + 1, nmod))
    ca = rng.normal(size=(2, nz2 + 1, nmod)) + 1j * rng.normal(size=(2, nz2 + 1, nmod))
    xs = np.arange(0, nx + 1) * dx               # psi nodes i = 0..nx
    arg = 2 * np.pi * xs[None, None, None, :] / lam[..., None] + ph[..., None]
    rx = (ca[..., None] * np.cos(arg)).sum(axis=2)   # (2, nz2+1, nx+1)

    u = np.zeros((nx, ny + 1, nz2 + 1), dtype=np.complex128)
    v = np.zeros((nx, ny, nz2 + 1), dtype=np.complex128)
    w = np.zeros((nx, ny + 1, nz2 + 1), dtype=np.complex128)
    # (u', v') from psi at the v nodes (y(j), x_i), psi(1) = psi(ny) = 0:
    #   u(j+1, i) = (psi(j+1,i) - psi(j,i))/dy(j), v(j,i) = -(psi(j,i)-psi(j,i-1))/dx
    psi = spec[None, :, None] * rx[0].T[:, :, None] * window(yv)[None, None, :]
    psi = np.transpose(psi, (0, 2, 1))            # (nx+1, ny, nz2+1)
    u[:, 1:ny, :] += (psi[1:, 1:, :] - psi[1:, :-1, :]) / dy[1:ny][None, :, None]
    v[:, :, :] += -(psi[1:, :, :] - psi[:-1, :, :]) / dx
    # (v', w') from phi at the v nodes: v(j) = i kz phi(j), w(j+1) = -(phi(j+1)-phi(j))/dy(j)
    phi = spec[None, :, None] * rx[1].T[1:, :, None] * window(yv)[None, None, :]
    phi = np.transpose(phi, (0, 2, 1))            # (nx, ny, nz2+1)
    v += 1j * kz[None, None, :] * phi
    w[:, 1:ny, :] += -(phi[:, 1:, :] - phi[:, :-1, :]) / dy[1:ny][None, :, None]
    pert = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max(), 1e-300)
    scale = cfg.amp / pert
    u *= scale
    v *= scale
    w *= scale
    u[:, :, 0] += U
    v[:, :, 0] += V
    u[0] = 0.0                                    # inflow plane: mean only
    u[0, :, 0] = U[0]
    v[0] = 0.0
    v[0, :, 0] = V[0]
    w[0] = 0.0

    def pack(c):
        r = np.empty(c.shape[:-1] + (2 * c.shape[-1],))
        r[..., 0::2] = c.real
        r[..., 1::2] = c.imag
        return r.astype(np.float32).astype(np.float64)

    uu, vv, ww = pack(u), pack(v), pack(w)
    xout = cfg.resolved_xout()
    return dict(
        u=uu, v=vv, w=ww,
        p=np.zeros((nx, ny, nz1)),
        rhsupa=np.zeros((nx, ny + 1, nz1)),
        rhsvpa=np.zeros((nx, ny, nz1)),
        rhswpa=np.zeros((nx, ny + 1, nz1)),
        y=y, re=re, xout=xout,
        u0=uu[0, :, 0].copy(), v0=vv[0, :, 0].copy(),
        um=uu[xout - 1, :, 0].copy(),
    )


def inlet_state(cfg: BoxConfig, base: dict) -> dict:
    """The fields of `base` (a state of the same grid size) as the initial
    state of box `cfg`: the fields and inlet profiles are shared, the
    Reynolds number, the recycling plane and its mean profile um are the
    box's own (a restart of a related run, as a serving client uploads it)."""
    y = y_grid(cfg)
    xout = cfg.resolved_xout()
    d = dict(base)
    d.update(y=y, re=reynolds_for(cfg, y), xout=xout, um=base["u"][xout - 1, :, 0].copy())
    return d
