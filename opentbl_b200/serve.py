"""Serving loop for 'advance this box by K RK3 steps' requests (no
counterpart in the reference, which runs one box per MPI job).

Continuous batching on one GPU: requests arrive at their own times (Poisson
arrivals in `make_requests`), wait in a FIFO queue, and are admitted as soon
as a slot and device memory are free under an HBM budget; every admitted
request owns a slot (a context: its own stream and device buffers) and runs
in chunks of RK3 steps, each chunk one CUDA graph launch, so the kernels of
all admitted requests overlap on the device. Slots are kept when their
request finishes and re-bound (otbl_ctx_rebind) to the next request of the
same grid size and precision; idle slots of other sizes are released when
memory is needed. A slot is prepared for its request on a background host
thread (a new context: device allocation, coefficient upload, autotuning;
or an idle one re-bound: the request's coefficients and initial fields
uploaded on the slot's stream; then the capture of its chunk's CUDA graph),
so the loop keeps feeding the running requests meanwhile. The host loop
never blocks on the device:
it polls each slot (otbl_query / otbl_graph_query) and issues the next chunk
when the last one has finished.

A request's result does not depend on the mix it ran in: its slot's kernels
read and write only the slot's buffers, on the slot's stream, and every
kernel is deterministic (tests/test_serve.py checks alone == in a mix, bit
for bit).
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import native, synth
from .box import Box
from .config import BoxConfig
from .ensemble import NX, NY, NZ, Graph


@dataclasses.dataclass
class Request:
    rid: int
    cfg: BoxConfig
    steps: int
    arrival: float  # seconds after the start of the run


@dataclasses.dataclass
class Result:
    rid: int
    name: str
    steps: int
    mpts: float
    arrival: float
    admitted: float
    finished: float
    dt: float = 0.0
    utauout: float = 0.0
    rthout: float = 0.0
    fields: dict | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def wait(self) -> float:
        return self.admitted - self.arrival


def make_requests(n: int, seed: int = 7, rate: float = 1.0, kmin: int = 10, kmax: int = 200,
                  large_frac: float = 0.1, precision: int = 1,
                  large: tuple = (1025, 193, 256)) -> list[Request]:
    """n requests with Poisson arrivals at `rate` per second and K ~ U[kmin,
    kmax]; sizes drawn as the ensemble sweep (nx in {129, 257, 385, 513}, ny
    in {65, 97, 129}, nz in {64, 128, 256}, Re_theta ~ U[300, 1500], Lx ~
    U[40, 80], Lz ~ U[6, 10]) with a fraction `large_frac` at `large`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        if rng.uniform() < large_frac:
            nx, ny, nz = large
        else:
            nx, ny, nz = int(rng.choice(NX)), int(rng.choice(NY)), int(rng.choice(NZ))
        rt = float(rng.uniform(300.0, 1500.0))
        cfg = BoxConfig(nx=nx, ny=ny, nz=nz, lx=float(rng.uniform(40.0, 80.0)), ly=8.0,
                        lz=float(rng.uniform(6.0, 10.0)), dy_wall=0.002, re_theta=rt,
                        profile="blasius" if rt < 700.0 else "musker", precision=precision,
                        name=f"req{k:04d}-{nx}x{ny}x{nz}")
        out.append(Request(rid=k, cfg=cfg, steps=int(rng.integers(kmin, kmax + 1)), arrival=t))
    return out


def size_key(cfg: BoxConfig) -> tuple:
    return (cfg.nx, cfg.ny, cfg.nz, cfg.precision)


class Templates:
    """Initial fields, one seeded synthetic field per grid size (the client's
    upload): a request starts from the field of its size class, generated at
    a class reference (Re_theta 1000, Lx 60, Lz 8) and cached; its
    coefficients follow its own Re_theta, Lx and Lz."""

    def __init__(self):
        self.cache = {}

    def get(self, cfg: BoxConfig) -> dict:
        key = (cfg.nx, cfg.ny, cfg.nz)
        if key not in self.cache:
            ref = dataclasses.replace(cfg, lx=60.0, lz=8.0, re_theta=1000.0, profile="musker",
                                      seed=1000003 * cfg.nx + 1009 * cfg.ny + cfg.nz)
            self.cache[key] = synth.make_initial(ref)
        base = self.cache[key]
        # the request's own inlet profile and recycling plane
        own = synth.inlet_state(cfg, base)
        return own

    def prepare(self, requests):
        for r in requests:
            self.get(r.cfg)


class _Slot:
    def __init__(self, box: Box, nbytes: int):
        self.box = box
        self.nbytes = nbytes
        self.req = None
        self.remaining = 0
        self.graph = None
        self.chunk = 0
        self.admitted = 0.0

    @property
    def key(self):
        return size_key(self.box.cfg)


class Server:
    def __init__(self, device: int = 0, budget_bytes: float = 150e9, chunk: int = 4,
                 max_active: int = 64, autotune: bool = True, keep_fields: bool = False,
                 templates: Templates | None = None):
        self.device = device
        self.budget = budget_bytes
        self.chunk = chunk
        self.max_active = max_active
        self.autotune = autotune
        self.keep_fields = keep_fields
        self.templates = templates or Templates()
        self.L = native.lib()
        self.idle = {}
        self.used = 0
        self.tuning = {}  # CTA sizes picked by the autotuner, per grid size
        self.creator = ThreadPoolExecutor(max_workers=1)
        self.pending = None  # (request, future of its new slot)
        self.stats = {"created": 0, "reused": 0, "evicted": 0, "graph_launches": 0,
                      "direct_steps": 0, "peak_bytes": 0, "peak_active": 0,
                      "create_s": 0.0, "rebind_s": 0.0, "capture_s": 0.0}

    # ---- slots ----
    def _bytes(self, cfg, init) -> int:
        c = native.make_config(cfg, init["re"], init["xout"])
        return int(self.L.otbl_ctx_bytes(c))

    def _evict_one(self) -> bool:
        for key, lst in self.idle.items():
            if lst:
                s = lst.pop()
                s.box.close()
                self.used -= s.nbytes
                self.stats["evicted"] += 1
                return True
        return False

    def _prepare(self, req: Request, init: dict, slot: "_Slot | None", need: int, key):
        """Runs on the preparation thread: a new context for req, autotuned
        (or given the CTA sizes already picked for its grid size), or the
        idle `slot` re-bound to req; then the CUDA graph of its chunk."""
        t = time.perf_counter()
        if slot is None:
            box = Box(req.cfg, init, device=self.device)
            if self.autotune:
                if key in self.tuning:
                    box.set_tuning(self.tuning[key])
                else:
                    self.tuning[key] = box.autotune()
            slot = _Slot(box, need)
            self.stats["create_s"] += time.perf_counter() - t
        else:
            slot.box.rebind(req.cfg, init)
            self.stats["rebind_s"] += time.perf_counter() - t
        t = time.perf_counter()
        slot.chunk = min(self.chunk, req.steps)
        slot.graph = Graph([slot.box], slot.chunk) if req.steps >= slot.chunk else None
        self.stats["capture_s"] += time.perf_counter() - t
        return slot

    def _acquire(self, req: Request, init: dict):
        """A slot for the request at the head of the queue, prepared in the
        background: an idle slot of its grid size re-bound, or a new one
        (None until it is ready, or while memory is short)."""
        key = size_key(req.cfg)
        if self.pending is not None:
            preq, fut, created = self.pending
            if preq is not req or not fut.done():
                return None
            self.pending = None
            self.stats["created" if created else "reused"] += 1
            return fut.result()
        lst = self.idle.get(key)
        if lst:
            s = lst.pop()
            self.pending = (req, self.creator.submit(self._prepare, req, init, s, s.nbytes, key), False)
            return None
        need = self._bytes(req.cfg, init)
        while self.used + need > self.budget and self._evict_one():
            pass
        if self.used + need > self.budget:
            return None
        self.used += need
        self.stats["peak_bytes"] = max(self.stats["peak_bytes"], self.used)
        self.pending = (req, self.creator.submit(self._prepare, req, init, None, need, key), True)
        return None

    def _issue(self, s: _Slot):
        """Next chunk of the slot's request: a graph launch of `chunk` steps,
        or the remainder as direct launches."""
        if s.remaining >= s.chunk and s.graph is not None:
            s.graph.launch()
            s.remaining -= s.chunk
            self.stats["graph_launches"] += 1
        else:
            n = s.remaining
            s.box.advance(n)
            s.remaining = 0
            self.stats["direct_steps"] += n

    def _busy(self, s: _Slot) -> bool:
        return (s.graph is not None and s.graph.busy()) or s.box.busy()

    def _finish(self, s: _Slot, now: float) -> Result:
        if s.graph is not None:
            s.graph.sync()
            s.graph.close()
            s.graph = None
        s.box.sync()
        _, inf = s.box.inflow()
        r = s.req
        res = Result(rid=r.rid, name=r.cfg.name, steps=r.steps, mpts=r.cfg.mpts, arrival=r.arrival,
                     admitted=s.admitted, finished=now, dt=inf["dt"], utauout=inf["utauout"],
                     rthout=inf["rthout"])
        if self.keep_fields:
            res.fields = {n: s.box.field(n) for n in native.FIELDS}
        s.req = None
        self.idle.setdefault(s.key, []).append(s)
        return res

    # ---- the loop ----
    def run(self, requests: list[Request], poll: float = 2e-4) -> list[Result]:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue = deque()
        active = []
        results = []
        head = None  # the queue head and its initial state
        t0 = time.perf_counter()
        while pending or queue or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            did = False
            # admission, first come first served
            while queue and len(active) < self.max_active:
                req = queue[0]
                if head is None or head[0] is not req:
                    head = (req, self.templates.get(req.cfg))
                init = head[1]
                s = self._acquire(req, init)
                if s is None:
                    break
                queue.popleft()
                s.req = req
                s.remaining = req.steps
                s.admitted = time.perf_counter() - t0
                active.append(s)
                self._issue(s)
                did = True
            self.stats["peak_active"] = max(self.stats["peak_active"], len(active))
            # progress: every slot whose last chunk has finished gets its next
            for s in list(active):
                if self._busy(s):
                    continue
                if s.remaining > 0:
                    self._issue(s)
                else:
                    active.remove(s)
                    results.append(self._finish(s, time.perf_counter() - t0))
                did = True
            if not did:
                if not active and not queue and pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                else:
                    time.sleep(poll)
        self.makespan = time.perf_counter() - t0
        return sorted(results, key=lambda r: r.rid)

    def close(self):
        self.creator.shutdown(wait=True)
        for lst in self.idle.values():
            for s in lst:
                s.box.close()
        self.idle = {}
        self.used = 0


def summarize(results: list[Result], makespan: float) -> dict:
    lat = np.array([r.latency for r in results])
    work = sum(r.mpts * 3 * r.steps for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "max_s": float(lat.max()), "mean_wait_s": float(np.mean([r.wait for r in results])),
            "makespan_s": makespan, "throughput": work / makespan,
            "unit": "Mpts·substeps/s"}
