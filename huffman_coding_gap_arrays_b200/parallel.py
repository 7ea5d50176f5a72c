"""Multi-GPU: a batch of independent buffers shards across ranks by bytes.

Buffers are independent (each has its own codebook and stream), so the
batched path needs no collective on its data path: every rank compresses
and decompresses its own share, one process per GPU.  The only exchanges
are the launch-time agreement on the partition (computed identically on
every rank from the sizes, no message), the max-over-ranks of the device
time, and -- if a caller wants every result on one rank -- a gather of the
finished containers.
"""
from __future__ import annotations

import heapq

import torch
import torch.distributed as dist


def shard_by_bytes(sizes, world: int) -> list:
    """Deterministic partition of buffer indices over `world` ranks that
    balances bytes: largest buffers first, each to the least-loaded rank
    (ties to the lowest rank); each rank's indices ascend."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over the process group (the slowest rank's time)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict, dst: int = 0):
    """Gathers {buffer index: bytes} from every rank to rank `dst`; returns
    the merged dict there (None elsewhere).  Off the timed path."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    out = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(local, out, dst=dst)
    if dist.get_rank() != dst:
        return None
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"buffer {k} produced by two ranks")
            merged[k] = v
    return merged


__all__ = ["shard_by_bytes", "max_over_ranks", "gather_results"]
