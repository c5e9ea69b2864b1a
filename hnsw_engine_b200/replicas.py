"""Host logic of multi-GPU search: one process per GPU, each with a full replica of the graph.

Queries are independent and the graph is read-only, so the search shards by query with no
collective on the data path. Each rank searches its own queries on its own replica. The only
exchanges are host-side:

* the maximum of the ranks' device timings, which makes a job's time the slowest rank's;
* optionally, gathering the ranks' result slices when one batch is split across GPUs.

Sharding the graph itself, with a k-way merge of per-shard results, would change results against
the reference's single graph, so it is not offered.

Everything here works with any ``torch.distributed`` backend: NCCL on GPUs, and gloo on CPU for
tests.
"""

from __future__ import annotations

import os
from typing import Any

import numpy as np


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment (1 process if unset)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} for world size {world}")
    return rank, world, local


def query_slice(nq: int, rank: int, world: int) -> slice:
    """Contiguous share of ``nq`` queries for ``rank``. Shares differ by at most one query, and the
    ranks' slices in rank order tile ``range(nq)``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} for world size {world}")
    base, extra = divmod(nq, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(dist: Any, value: float, device: Any = "cpu") -> float:
    """Maximum of ``value`` over all ranks (``dist`` is ``torch.distributed`` or None for 1 rank)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, units_per_rank: int, steps: int, total_ms: float) -> float:
    """Units per second of the whole job. Every rank processes ``units_per_rank`` per step, and
    ``total_ms`` is the slowest rank's time for ``steps`` steps."""
    if total_ms <= 0:
        raise ValueError("total_ms must be positive")
    return world * units_per_rank * steps / (total_ms / 1000.0)


def gather_results(dist: Any, ids: np.ndarray, dists: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Concatenate every rank's (ids, dists) slices in rank order. Every rank receives the
    concatenation. The slices are host arrays whose first dimension is the query."""
    if dist is None:
        return ids, dists
    parts: list[Any] = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (np.ascontiguousarray(ids), np.ascontiguousarray(dists)))
    return (np.concatenate([p[0] for p in parts], axis=0),
            np.concatenate([p[1] for p in parts], axis=0))
