"""Shared test helpers: box setup for the product and the oracle on the same
seeded inputs and the same coefficient bits."""
import numpy as np

from opentbl_b200 import config, native, synth
from oracle import pyoracle


def setup(cfg):
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    return init, coef


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


def max_abs(a):
    return float(np.max(np.abs(a)))


def oracle_box(cfg, init, coef, threads=0):
    return pyoracle.OracleBox(cfg, init, coef, threads=threads)


def divergence_np(cfg, coef, u, v, w):
    """pois.f90:41-54 in numpy on (nx, rows, nz1) arrays; rows 1..ny-1 of
    planes 2..nx (other entries 0)."""
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
