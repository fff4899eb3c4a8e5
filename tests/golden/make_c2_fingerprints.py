"""Writes tests/golden/c2_oracle_fingerprints.npz: fingerprints of the
oracle's state on the seeded 1025x193x512 box (Re_theta 1000, FP64,
adaptive dt) after 20 and 100 RK3 steps.

The oracle needs about half an hour of host time for the 100 steps, far too
long for a test, so the GPU tests compare against these stored fingerprints
instead of a fresh oracle run. Each checkpoint stores quantities that cover
the whole field (so a local error cannot hide) and point values:

  norm_<f>      Parseval-weighted L2 norm of u, v, w, p (k = 0 weight 1,
                k > 0 weight 2, as stotf.F90:155)
  plane_<f>     the same per streamwise plane (nx values) for u, v, w
  mode_<f>      the same per spanwise mode (nz2+1 values) for u, v, w
  meanU         Re u(k=0) averaged over the planes, per row (ny+1)
  Uxout         Re u(k=0) at plane xout, per row (ny+1)
  um            the filtered mean profile of genflu (ny+1)
  vals_<f>      the values at 2048 seeded flat indices idx_<f>, for u, v, w, p
  scal          tiempo, dt, utauout, rthout, dout, gamma1, gamma2, timec
  ener          the 15 energies of rhsp (last substep 1)
  divmax        max |div u| (pois.f90:41-54) after the last projection

    python tests/golden/make_c2_fingerprints.py [threads]
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from opentbl_b200 import config, synth  # noqa: E402
from oracle import pyoracle  # noqa: E402

OUT = os.path.join(HERE, "c2_oracle_fingerprints.npz")
CHECKPOINTS = (20, 100)
SCALARS = ("tiempo", "dt", "utauout", "rthout", "dout", "gamma1", "gamma2", "timec")
NSAMPLE = 2048


def parseval_weights(nz1):
    w = np.full(nz1, 2.0)
    w[:2] = 1.0            # k = 0 (real and imaginary slot)
    return w


def sample_index(shape, field):
    rng = np.random.default_rng({"u": 11, "v": 12, "w": 13, "p": 14}[field])
    return np.sort(rng.choice(int(np.prod(shape)), size=NSAMPLE, replace=False))


def fingerprints(cfg, fields, um, st, ener, divmax):
    out = {}
    w = parseval_weights(cfg.nz1)
    for f, a in fields.items():
        sq = a * a * w
        out[f"norm_{f}"] = np.array([np.sqrt(sq.sum())])
        if f in "uvw":
            out[f"plane_{f}"] = np.sqrt(sq.sum(axis=(1, 2)))
            out[f"mode_{f}"] = np.sqrt(sq.reshape(cfg.nx, -1, cfg.nz1 // 2, 2).sum(axis=(0, 1, 3)))
        idx = sample_index(a.shape, f)
        out[f"idx_{f}"] = idx
        out[f"vals_{f}"] = a.ravel()[idx]
    u = fields["u"]
    out["meanU"] = u[:, :, 0].mean(axis=0)
    out["Uxout"] = u[cfg.resolved_xout() - 1, :, 0].copy()
    out["um"] = np.asarray(um, dtype=np.float64)
    out["scal"] = np.array([st[k] for k in SCALARS])
    out["ener"] = np.asarray(ener, dtype=np.float64)
    out["divmax"] = np.array([divmax])
    return out


def make(threads: int = 0):
    cfg = config.C2
    init = synth.make_initial(cfg)
    ob = pyoracle.OracleBox(cfg, init, threads=threads)
    res = {}
    done = 0
    t0 = time.time()
    for target in CHECKPOINTS:
        for _ in range(target - done):
            ob.advance(1)
            done += 1
            print(f"step {done} ({time.time() - t0:.0f} s)", flush=True)
        fields = {f: ob.field(f) for f in ("u", "v", "w", "p")}
        um, st = ob.inflow()
        divmax = float(np.abs(ob.divergence()).max())
        fp = fingerprints(cfg, fields, um, st, ob.energies(), divmax)
        for k, v in fp.items():
            res[f"s{target}_{k}"] = v
        print(f"checkpoint {target}: divmax {divmax:.3e}, rthout {st['rthout']:.6f}", flush=True)
    ob.close()
    res["meta"] = np.array(json.dumps({"config": cfg.name, "checkpoints": list(CHECKPOINTS),
                                       "scalars": list(SCALARS), "nsample": NSAMPLE,
                                       "seconds": time.time() - t0}))
    np.savez_compressed(OUT, **res)
    print("wrote", OUT)


if __name__ == "__main__":
    make(int(sys.argv[1]) if len(sys.argv) > 1 else 0)
