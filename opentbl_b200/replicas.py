"""Replica placement for independent boxes, one process per GPU.

A single box does not shard without the reference's global transposes
(change.f90 x-slab <-> pencil all-to-all), so multi-GPU runs are replicas:
every rank advances its own box on its own device, with no collective on the
data path. The only collectives are the barrier around the timed region and
the max over ranks of the elapsed time. The backend is NCCL when CUDA is
available and gloo otherwise (CPU tests with world_size > 1).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Rank:
    world_size: int
    rank: int
    local_rank: int
    backend: str | None = None

    @property
    def device(self) -> int:
        return self.local_rank


def setup(backend: str | None = None, timeout_s: float = 300.0) -> Rank:
    """Reads WORLD_SIZE/RANK/LOCAL_RANK (torchrun) and joins the group when
    world_size > 1."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    r = Rank(ws, rank, local)
    if ws > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
        r.backend = backend
    return r


def max_over_ranks(x: float, r: Rank) -> float:
    if r.world_size == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if r.backend == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(r: Rank):
    if r.world_size > 1:
        import torch.distributed as dist
        dist.barrier()


def aggregate_rate(units_per_rank: float, seconds_max: float, r: Rank) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return r.world_size * units_per_rank / seconds_max


def teardown(r: Rank):
    if r.world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
