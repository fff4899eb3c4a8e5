"""Ensembles (one CUDA graph over many boxes), the autotuner and the serving
loop. CPU tests cover request generation and the host logic of admission;
GPU tests check that a graph-launched ensemble and the serving mix give the
same bits as each box advanced alone."""
import numpy as np
import pytest

from opentbl_b200 import Box, config, ensemble, native, serve, synth
from opentbl_b200.config import replace


def test_requests_are_seeded_and_poisson():
    a = serve.make_requests(200, seed=3, rate=5.0)
    b = serve.make_requests(200, seed=3, rate=5.0)
    assert [(r.cfg, r.steps, r.arrival) for r in a] == [(r.cfg, r.steps, r.arrival) for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 0.2) < 0.05
    assert all(10 <= r.steps <= 200 for r in a)
    big = sum(1 for r in a if (r.cfg.nx, r.cfg.ny, r.cfg.nz) == (1025, 193, 256))
    assert 5 <= big <= 40


def test_ensemble_configs_are_valid():
    L = native.lib()
    for c in ensemble.ensemble_configs(24):
        init = synth.make_initial(replace(c, nx=c.nx)) if c.nx <= 129 and c.nz <= 64 else None
        y = synth.y_grid(c)
        re = synth.reynolds_for(c, y)
        cc = native.make_config(c, re, c.resolved_xout())
        assert L.otbl_config_check(cc) == 0, c.name
        assert L.otbl_ctx_bytes(cc) > 0
        if init is not None:
            assert init["u"].shape == (c.nx, c.ny + 1, c.nz1)


def test_ctx_bytes_grows_with_the_box_and_mixed_is_smaller():
    L = native.lib()
    a = native.make_config(config.C1, 1000.0, 20)
    b = native.make_config(config.C2, 1000.0, 100)
    m = native.make_config(replace(config.C2, precision=1), 1000.0, 100)
    assert 0 < L.otbl_ctx_bytes(a) < L.otbl_ctx_bytes(b)
    assert L.otbl_ctx_bytes(m) < L.otbl_ctx_bytes(b)
    # 1025x193x512 FP64: 7 state + 15 intermediates + 6 scratch fields (the
    # w tail runs beside the v tail on a scratch set of its own)
    nf = 1025 * 194 * 340 * 8
    assert 28 * nf <= L.otbl_ctx_bytes(b) <= 29.5 * nf


class _FakeBox:
    """Host stand-in for Box in the admission logic (no device)."""
    def __init__(self, cfg):
        self.cfg = cfg
        self.closed = False

    def close(self):
        self.closed = True


def test_admission_evicts_idle_slots_of_other_sizes():
    srv = serve.Server.__new__(serve.Server)
    srv.budget, srv.used, srv.idle = 10, 0, {}
    srv.stats = {"evicted": 0}
    boxes = [serve._Slot(_FakeBox(replace(config.TINY, nx=n)), 4) for n in (33, 41)]
    for s in boxes:
        srv.idle.setdefault(s.key, []).append(s)
        srv.used += s.nbytes
    assert srv._evict_one() and srv.used == 4 and srv.stats["evicted"] == 1
    assert srv._evict_one() and srv.used == 0
    assert not srv._evict_one()
    assert all(b.box.closed for b in boxes)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_ctx_bytes_is_what_a_context_allocates(precision):
    """The admission estimate is exact: otbl_ctx_bytes equals the device
    bytes a context of that configuration holds."""
    cfg = replace(config.TINY, precision=precision)
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    b = Box(cfg, init, coef)
    cc = native.make_config(cfg, init["re"], init["xout"])
    assert b.device_bytes == native.lib().otbl_ctx_bytes(cc)
    b.close()


@pytest.mark.gpu
def test_graph_ensemble_equals_boxes_alone():
    """Three boxes of different sizes and both precisions in one CUDA graph
    (two launches of 2 RK3 steps) against each box advanced alone."""
    cfgs = [config.TINY, replace(config.SMALL, precision=1), replace(config.TINY, nx=49, nz=64, precision=1)]
    inits = [synth.make_initial(c) for c in cfgs]
    alone = []
    for c, i in zip(cfgs, inits):
        b = Box(c, i)
        b.advance(4)
        alone.append({n: b.field(n) for n in native.FIELDS})
        b.close()
    boxes = [Box(c, i) for c, i in zip(cfgs, inits)]
    for b in boxes:
        b.autotune()
    g = ensemble.Graph(boxes, 2)
    assert g.kernels > 0
    l0 = [b.launches for b in boxes]
    g.launch()
    g.launch()
    g.sync()
    assert sum(b.launches - l for b, l in zip(boxes, l0)) == 2 * g.kernels
    for b, ref in zip(boxes, alone):
        for n in native.FIELDS:
            assert np.array_equal(b.field(n), ref[n]), (b.cfg.name, n)
    g.close()
    for b in boxes:
        b.close()


@pytest.mark.gpu
def test_serving_mix_equals_alone():
    """Six requests on three grid sizes (slots are created, re-bound and
    reused), arriving while others run: each result equals the same request
    served alone, bit for bit."""
    reqs = serve.make_requests(6, seed=11, rate=50.0, kmin=3, kmax=7, large_frac=0.0)
    for r in reqs:
        r.cfg = replace(r.cfg, nx=[33, 49, 65][r.rid % 3], ny=41, nz=32, lx=12.0, ly=6.0,
                        lz=4.0, dy_wall=0.02, re_theta=300.0 + 50 * r.rid, profile="blasius",
                        xout=0)
    tpl = serve.Templates()
    # two slots at most: later arrivals queue, then re-bind a finished slot
    srv = serve.Server(budget_bytes=2e9, chunk=2, max_active=2, keep_fields=True, templates=tpl)
    mix = srv.run(reqs)
    assert srv.stats["reused"] >= 1 and srv.stats["peak_active"] >= 2
    srv.close()
    for r in reqs:
        one = serve.Server(budget_bytes=2e9, chunk=2, keep_fields=True, templates=tpl)
        res = one.run([serve.Request(r.rid, r.cfg, r.steps, 0.0)])[0]
        one.close()
        for n in native.FIELDS:
            assert np.array_equal(res.fields[n], mix[r.rid].fields[n]), (r.rid, n)
    s = serve.summarize(mix, srv.makespan)
    assert s["requests"] == 6 and s["p99_s"] >= s["p50_s"] > 0


@pytest.mark.gpu
def test_bounded_device_wait_reports_timeout():
    """The bounded mbarrier wait of the TMA-fed kernels on a barrier that
    never completes: the kernel gives up after 1 ms and reports
    OTBL_ERR_TIMEOUT; the context keeps working afterwards."""
    import ctypes
    cfg = config.TINY
    init = synth.make_initial(cfg)
    b = Box(cfg, init)
    st = ctypes.c_int(0)
    assert b.L.otbl_selftest_wait(b.h, ctypes.byref(st)) == native.OTBL_OK
    assert st.value == 8  # OTBL_ERR_TIMEOUT
    b.advance(1)
    b.sync()
    assert np.isfinite(b.field("u")).all()
    b.close()
