"""Host-side diagnostics of a box state (numpy): the divergence that pois
removes (pois.f90:41-54) and the error measures used to compare two runs."""
from __future__ import annotations

import numpy as np

from . import native


def divergence(cfg, coef, u, v, w):
    """pois.f90:41-54 on (nx, rows, nz1) plane-layout arrays: complex
    divergence of rows 1..ny-1 of planes 2..nx (other entries 0)."""
    off = native.coef_offsets(cfg)
    nz2 = cfg.nz2
    kaz = coef[off["KAZ"]:off["KAZ"] + nz2 + 1]
    idy = coef[off["IDY"]:off["IDY"] + cfg.ny + 1]
    idx = coef[off["SCAL"] + native.SCAL["IDX"]]
    uc = u[..., 0::2] + 1j * u[..., 1::2]
    vc = v[..., 0::2] + 1j * v[..., 1::2]
    wc = w[..., 0::2] + 1j * w[..., 1::2]
    ny = cfg.ny
    d = np.zeros((cfg.nx, ny, nz2 + 1), dtype=np.complex128)
    j = np.arange(1, ny)  # rows 1..ny-1
    d[1:, :ny - 1] = (wc[1:, j] * (1j * kaz)[None, None, :]
                      + (vc[1:, j] - vc[1:, j - 1]) * idy[j][None, :, None])
    d[1:, :ny - 1] = d[1:, :ny - 1] + idx * (uc[1:, j] - uc[:-1, j])
    return d


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def velocity_rel_l2(g, o):
    """Relative L2 of the velocity over u, v, w together, Parseval-weighted
    (mode k = 0 counted once, k > 0 twice, as stotf.F90:155); g and o map
    "u", "v", "w" to (nx, rows, nz1) arrays."""
    num = den = 0.0
    for n in "uvw":
        a, b = np.asarray(g[n]), np.asarray(o[n])
        wgt = np.full(a.shape[-1], 2.0)
        wgt[:2] = 1.0
        num += float((((a - b) ** 2) * wgt).sum())
        den += float(((b ** 2) * wgt).sum())
    return (num / den) ** 0.5


def compare(cfg, coef, box, ref) -> dict:
    """Error of `box` against `ref` (two Box-like objects on the same grid):
    velocity L2, max|div u| of `box`, mean profile U(y) = Re u(k=0) at xout,
    the filtered mean um, Re_theta and C_f = 2 u_tau^2 (genflu.F90:76-87)."""
    gv = {n: box.field(n) for n in "uvw"}
    ov = {n: ref.field(n) for n in "uvw"}
    um_g, gi = box.inflow()
    um_o, oi = ref.inflow()
    x = cfg.resolved_xout() - 1
    return {
        "vel_rel_l2": velocity_rel_l2(gv, ov),
        "max_div": float(np.abs(divergence(cfg, coef, gv["u"], gv["v"], gv["w"])).max()),
        "U_rel_l2": rel_l2(gv["u"][x, :, 0], ov["u"][x, :, 0]),
        "um_rel_l2": rel_l2(um_g, um_o),
        "re_theta_rel": abs(gi["rthout"] - oi["rthout"]) / abs(oi["rthout"]),
        "cf_rel": abs(gi["utauout"] ** 2 - oi["utauout"] ** 2) / oi["utauout"] ** 2,
    }
