"""Multi-GPU replicas: one process per GPU, each with its own copy of the
index and its own share of the queries. The hot path has no exchange step,
so nothing crosses NVLink on the data path; the only collectives are the
host-side barrier and the max-over-ranks of the timings.

The reference is single-GPU (one caller stream, no NCCL or MPI anywhere);
this module has no reference counterpart.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) share of n items for rank (sizes differ by <= 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    b = rank * base + min(rank, extra)
    return b, b + base + (1 if rank < extra else 0)


def shard_queries(q_off: np.ndarray, q_terms: np.ndarray, rank: int, world: int):
    """This rank's queries as (offsets rebased to 0, terms, first query index)."""
    n = q_off.size - 1
    a, b = shard_range(n, rank, world)
    off = (q_off[a:b + 1] - q_off[a]).astype(np.uint64)
    return off, q_terms[q_off[a]:q_off[b]], a


def rank_seed(base: int, rank: int) -> int:
    """Query-set seed of a rank in weak-scaling runs (every rank its own queries)."""
    return int(base) + 1000 * int(rank)


def max_over_ranks(x: float, dist=None) -> float:
    """Max of a host float over the process group (identity without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
