"""Multi-GPU counting by replicas: colorings are independent, so each rank
counts its own contiguous share of them on its own GPU (one process per GPU)
and the FP64 raw counts are gathered in coloring order.  No count table or
aggregate crosses ranks; the only collective is the gather of n doubles.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np


def shard(n_colorings: int, world: int, rank: int) -> tuple[int, int]:
    """(first coloring, count) of `rank` in a contiguous block partition."""
    if world < 1 or not 0 <= rank < world or n_colorings < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n_colorings, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gather_raw(local: np.ndarray, n_colorings: int, group=None) -> np.ndarray:
    """All ranks' raw counts in coloring order (every rank receives them)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [shard(n_colorings, world, r)[1] for r in range(world)]
    width = max(counts) if counts else 0
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[: len(local)] = torch.from_numpy(np.ascontiguousarray(local, np.float64)).to(device)
    parts = [torch.zeros(width, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)])


def count_replicas(count_fn: Callable[[int, int], np.ndarray], n_colorings: int, seed_base: int,
                   group=None) -> np.ndarray:
    """Runs count_fn(first_seed, n) for this rank's colorings and gathers all raw counts.

    count_fn(seed, n) must return the raw counts of colorings seeded seed, seed+1, ...;
    with subgraph_b200 it is `lambda s, n: sg.count(graph, template, n, s)`.
    """
    import torch.distributed as dist
    if not dist.is_initialized():
        return np.asarray(count_fn(seed_base, n_colorings), np.float64)
    first, cnt = shard(n_colorings, dist.get_world_size(group), dist.get_rank(group))
    local = np.asarray(count_fn(seed_base + first, cnt), np.float64) if cnt else np.zeros(0)
    return gather_raw(local, n_colorings, group)


def estimate_replicas(raw: np.ndarray, k: int, automorphisms: int = 1, estimate_fn: Optional[Callable] = None) -> float:
    """The reference's final estimate over all gathered colorings."""
    if estimate_fn is None:
        from . import api
        estimate_fn = api.estimate
    return float(estimate_fn(raw, k, automorphisms))
