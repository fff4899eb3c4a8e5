"""Shared test helpers: box setup for the product and the oracle on the same
seeded inputs and the same coefficient bits."""
import numpy as np

from opentbl_b200 import config, diag, native, synth
from oracle import pyoracle


def setup(cfg):
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    return init, coef


rel_l2 = diag.rel_l2
velocity_rel_l2 = diag.velocity_rel_l2


def max_abs(a):
    return float(np.max(np.abs(a)))


def oracle_box(cfg, init, threads=0):
    """The oracle on the same seeded input; it computes its coefficients
    with its own set-up code (oracle/orc_coef.c)."""
    return pyoracle.OracleBox(cfg, init, threads=threads)


divergence_np = diag.divergence
