"""Multi-GPU plumbing: one process per GPU (torchrun), replicas or channel
shards with no data-path collective.

A single channel does not shard (its step has no exchange worth a
collective here): N GPUs run N independent channels.  A batch of channels
shards by channel: each rank takes a set of channels whose node counts sum
to nearly the same total, and the only collectives are the barrier and the
max of the ranks' timings around the timed region.
"""
from __future__ import annotations

import datetime
import os


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class Dist:
    """Rank, world size and the two collectives of the timing protocol.
    backend: "nccl" (GPU ranks) or "gloo" (CPU ranks, used by the tests)."""

    def __init__(self, use_pg=True, backend="nccl", timeout_s=120):
        self.world = _env_int("WORLD_SIZE", 1)
        self.rank = _env_int("RANK", 0)
        self.local = _env_int("LOCAL_RANK", 0)
        self.backend = backend
        self.pg = None
        if self.world > 1 and use_pg:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], device=dev, dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()
            self.pg = None


def shard_by_nodes(specs, world, rank):
    """Indices of the channels of `rank`: longest-processing-time-first over
    node counts (largest channel to the least loaded rank, ties to the lower
    rank), deterministic, every channel on exactly one rank."""
    order = sorted(range(len(specs)), key=lambda i: (-specs[i]["nx"] * specs[i]["ny"], i))
    load = [0] * world
    owner = {}
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += specs[i]["nx"] * specs[i]["ny"]
    return sorted(i for i, r in owner.items() if r == rank)
