"""The N > 1 path on CPU: world_size-2 gloo groups (127.0.0.1).

Multi-GPU runs are replicas (one independent box per rank, no collective on
the data path); these tests cover the host logic around them -- group setup,
the barrier, the max over ranks of the elapsed time, the whole-job rate --
with the oracle standing in for each rank's box, and bench.py's reference
arm under torchrun, where rank 0 alone measures and prints.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import time
    from opentbl_b200 import config, replicas
    from helpers import oracle_box, setup
    R = replicas.setup("gloo", timeout_s=60)
    init, coef = setup(config.TINY)
    ob = oracle_box(config.TINY, init, threads=1)
    replicas.barrier(R)
    t0 = time.perf_counter()
    ob.substep(1, 1)
    el = time.perf_counter() - t0 + 0.01 * rank   # ranks differ in time
    mx = replicas.max_over_ranks(el, R)
    rate = replicas.aggregate_rate(config.TINY.mpts, mx, R)
    q.put((rank, el, mx, rate, float(np.linalg.norm(ob.field("u"))), R.backend))
    replicas.barrier(R)
    replicas.teardown(R)


def test_two_gloo_replicas():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, e0, m0, v0, n0, b0), (r1, e1, m1, v1, n1, b1) = out
    assert b0 == b1 == "gloo"
    assert m0 == m1 == max(e0, e1)
    assert v0 == v1
    from opentbl_b200 import config
    assert abs(v0 - 2 * config.TINY.mpts / m0) <= 1e-12 * v0
    # independent boxes on the same seed: identical results, no cross-talk
    assert n0 == n1


def test_bench_reference_arm_under_torchrun():
    """bench.py --impl reference on 2 ranks: rank 0 prints one JSON line with
    the contract's keys, rank 1 exits 0 without work."""
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1", "--config", "TINY"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 1  # as asked (full RK3 steps)
    # the same workload config as the GPU arm, and nothing of the product loaded
    sys.path.insert(0, ROOT)
    import bench
    from opentbl_b200 import config
    assert d["config"] == bench.workload_config(config.TINY, 2)
    assert d["libraries_loaded"] == ["oracle/liboracle.so"], d["libraries_loaded"]
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
