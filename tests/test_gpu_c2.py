"""The headline box, 1025x193x512 (Re_theta 1000), after 20 and 100 RK3
steps against the oracle's fingerprints (tests/golden/c2_oracle_fingerprints.npz,
written by tests/golden/make_c2_fingerprints.py: the oracle needs half an
hour of host time for these steps).

FP64 path: the north star's gates, velocity relative L2 <= 1e-9 (here over
2048 seeded points per component and over the whole field's Parseval norms
per plane and per spanwise mode), max|div u| <= 1e-12, mean U(y), Re_theta
and C_f = 2 u_tau^2 to 1e-9.

Mixed path (OTBL_PREC_MIXED): velocity relative L2 <= 1e-5 and max|div u|
<= 1e-10 against the same FP64 oracle; its U(y), Re_theta and C_f errors are
printed and bounded at 1e-5.
"""
import json
import os

import numpy as np
import pytest

from opentbl_b200 import Box, config
from opentbl_b200.config import replace

from helpers import divergence_np, setup

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "c2_oracle_fingerprints.npz")


@pytest.fixture(scope="module")
def fx():
    d = np.load(FIX)
    meta = json.loads(str(d["meta"]))
    return d, meta


def _weights(nz1):
    w = np.full(nz1, 2.0)
    w[:2] = 1.0
    return w


def _compare(cfg, coef, g, d, meta, s):
    """Errors of the GPU state against checkpoint s of the fixture."""
    P = f"s{s}_"
    fields = {f: g.field(f) for f in ("u", "v", "w", "p")}
    w = _weights(cfg.nz1)
    num = den = 0.0
    out = {}
    for f in ("u", "v", "w"):
        a = fields[f]
        got = a.ravel()[d[P + "idx_" + f]]
        ref = d[P + "vals_" + f]
        num += float(np.sum((got - ref) ** 2))
        den += float(np.sum(ref ** 2))
        sq = a * a * w
        plane = np.sqrt(sq.sum(axis=(1, 2)))
        mode = np.sqrt(sq.reshape(cfg.nx, -1, cfg.nz1 // 2, 2).sum(axis=(0, 1, 3)))
        out[f"norm_{f}"] = abs(np.sqrt(sq.sum()) - d[P + "norm_" + f][0]) / d[P + "norm_" + f][0]
        out[f"plane_{f}"] = float(np.max(np.abs(plane - d[P + "plane_" + f]) / d[P + "plane_" + f].max()))
        out[f"mode_{f}"] = float(np.max(np.abs(mode - d[P + "mode_" + f]) / d[P + "mode_" + f].max()))
    out["vel_points"] = np.sqrt(num / den)
    pv = fields["p"].ravel()[d[P + "idx_p"]]
    out["p_points"] = float(np.linalg.norm(pv - d[P + "vals_p"]) / np.linalg.norm(d[P + "vals_p"]))
    u = fields["u"]
    for k, a in (("meanU", u[:, :, 0].mean(axis=0)),
                 ("Uxout", u[cfg.resolved_xout() - 1, :, 0])):
        out[k] = float(np.linalg.norm(a - d[P + k]) / np.linalg.norm(d[P + k]))
    um, st = g.inflow()
    out["um"] = float(np.linalg.norm(um - d[P + "um"]) / np.linalg.norm(d[P + "um"]))
    sc = dict(zip(meta["scalars"], d[P + "scal"]))
    out["rthout"] = abs(st["rthout"] - sc["rthout"]) / sc["rthout"]
    out["cf"] = abs(st["utauout"] ** 2 - sc["utauout"] ** 2) / sc["utauout"] ** 2
    out["tiempo"] = abs(st["tiempo"] - sc["tiempo"]) / sc["tiempo"]
    out["divmax"] = float(np.abs(divergence_np(cfg, coef, fields["u"], fields["v"], fields["w"])).max())
    out["divmax_oracle"] = float(d[P + "divmax"][0])
    return out


def _run(cfg, d, meta):
    init, coef = setup(cfg)
    g = Box(cfg, init, coef)
    res = {}
    done = 0
    for s in meta["checkpoints"]:
        g.advance(s - done)
        done = s
        res[s] = _compare(cfg, coef, g, d, meta, s)
        print(f"{cfg.name} prec={cfg.precision} after {s} steps:",
              {k: f"{v:.2e}" for k, v in res[s].items()})
    g.close()
    return res


def test_c2_fp64_against_oracle_fingerprints(fx):
    d, meta = fx
    res = _run(config.C2, d, meta)
    for s, e in res.items():
        assert e["vel_points"] <= 1e-9, (s, e)
        for f in "uvw":
            assert e[f"norm_{f}"] <= 1e-9 and e[f"plane_{f}"] <= 1e-9 and e[f"mode_{f}"] <= 1e-9, (s, f, e)
        assert e["p_points"] <= 1e-8, (s, e)
        for k in ("meanU", "Uxout", "um", "rthout", "cf"):
            assert e[k] <= 1e-9, (s, k, e)
        assert e["tiempo"] <= 1e-12, (s, e)
        assert e["divmax"] <= max(1e-12, 4 * e["divmax_oracle"]), (s, e)


def test_c2_mixed_against_oracle_fingerprints(fx):
    d, meta = fx
    res = _run(replace(config.C2, precision=1), d, meta)
    for s, e in res.items():
        assert e["vel_points"] <= 1e-5, (s, e)
        for f in "uvw":
            assert e[f"norm_{f}"] <= 1e-5 and e[f"plane_{f}"] <= 1e-5, (s, f, e)
        for k in ("meanU", "Uxout", "um", "rthout", "cf"):
            assert e[k] <= 1e-5, (s, k, e)
        assert e["divmax"] <= 1e-10, (s, e)
