"""Checkpoint files (escru.F90 escribezy/writeheader content, read back as
getstartzy/readheader do): container round trip on CPU; on the GPU a
checkpoint of a running box restarts into a new context and the next step
agrees with the oracle restarted from the same files."""
import math
import os

import numpy as np
import pytest

from opentbl_b200 import Box, checkpoint, config, native, synth

from helpers import oracle_box, rel_l2, setup


def test_container_round_trip_keeps_dtypes(tmp_path):
    a = np.arange(24, dtype=">f4").reshape(2, 3, 4)
    b = np.array([1.5], dtype="<f8")
    c = np.array([7], dtype="<i4")
    s = np.frombuffer(b"u", dtype="S1").copy()
    p = str(tmp_path / "x.otc")
    checkpoint.write_container(p, [("value", a), ("tiempo", b), ("nx", c), ("Variable", s)])
    d = checkpoint.read_container(p)
    assert d["value"].dtype == np.dtype(">f4") and np.array_equal(d["value"], a)
    assert d["tiempo"].dtype == np.dtype("<f8") and d["tiempo"][0] == 1.5
    assert d["nx"][0] == 7 and d["Variable"].tobytes() == b"u"
    with open(p, "rb") as f:
        assert f.read(8) == checkpoint.MAGIC


def test_file_names_follow_escribezy():
    assert checkpoint.file_name("run/bl", 7, "u") == "run/bl.007.u.otc"


class _HostBox:
    """Box-like holder of a synthetic state (no device)."""
    def __init__(self, cfg, init):
        self.cfg, self.init = cfg, init
        self.re, self.xout, self.y = init["re"], init["xout"], init["y"]

    def sync(self):
        pass

    def field(self, n):
        return self.init[n]

    def inflow(self):
        return self.init["um"], {"tiempo": 2.5, "timeinit": 0.5, "dt": 0.01}


def test_write_read_state_and_header(tmp_path):
    cfg = config.TINY
    init = synth.make_initial(cfg)
    init["p"] = np.random.default_rng(0).normal(size=init["p"].shape)
    hb = _HostBox(cfg, init)
    names = checkpoint.write(hb, str(tmp_path / "bl"), 3)
    assert [os.path.basename(n) for n in names] == [f"bl.003.{v}.otc" for v in "uvwp"]
    r = checkpoint.read(str(tmp_path / "bl"), 3)
    for n in "uvw":   # synthetic fields are FP32-representable
        assert np.array_equal(r[n], init[n])
    assert np.array_equal(r["p"], init["p"].astype(np.float32).astype(np.float64))
    assert not r["rhsupa"].any() and r["rhsvpa"].shape == init["rhsvpa"].shape
    assert r["tiempo"] == 2.5 and r["timeinit"] == 0.5 and r["dt"] == 0.01
    assert r["xout"] == init["xout"] and r["re"] == init["re"]
    assert np.array_equal(r["y"], init["y"]) and np.array_equal(r["um"], init["um"])
    assert math.isclose(r["lx"], cfg.ax * math.pi) and math.isclose(r["lz"], cfg.az * 2 * math.pi)
    assert np.array_equal(r["u0"], init["u"][0, :, 0])
    raw = checkpoint.read_container(str(tmp_path / "bl.003.v.otc"))
    assert raw["value"].dtype == np.dtype(">f4") and raw["value"].shape == (cfg.nx, cfg.ny, cfg.nz1)
    assert raw["nz2"][0] == cfg.nz2 and raw["procs"][0] == 1


@pytest.mark.gpu
def test_restart_continues_like_the_oracle(tmp_path):
    cfg = config.SMALL
    init, coef = setup(cfg)
    g = Box(cfg, init, coef)
    g.advance(2)
    checkpoint.write(g, str(tmp_path / "bl"), 1)
    r = checkpoint.read(str(tmp_path / "bl"), 1)
    h = Box(cfg, r, coef)
    for n in native.FIELDS:
        assert np.array_equal(h.field(n), r[n]), n
    o = oracle_box(cfg, r)
    h.advance(1)
    o.advance(1)
    for n in ("u", "v", "w", "p"):
        assert rel_l2(h.field(n), o.field(n)) <= 1e-10, n
    assert abs(h.inflow()[1]["tiempo"] - o.inflow()[1]["tiempo"]) <= 1e-14 * o.inflow()[1]["tiempo"]
