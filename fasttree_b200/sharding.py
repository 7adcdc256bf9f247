"""Query sharding of one tree across ranks (one process per GPU).

Self-kNN queries are independent: every rank holds the same tree (each rank builds it from
the same points -- the build is deterministic, so the trees are bit-identical -- or receives
it from one rank with broadcast_tree) and answers a contiguous range of sorted leaf ranks, i.e. a contiguous stretch of the
space-filling curve, so each rank's queries stay spatially coherent.  No collective is on
the data path; ranks only agree on the plan (computed identically everywhere) and reduce
their timings.

shard_ranges() balances the ranges by an optional per-query cost (for example the learned
bound's prediction or measured node visits); without costs the split is even.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np


def shard_ranges(num: int, world: int, costs: Optional[Sequence[float]] = None) -> List[Tuple[int, int]]:
    """Contiguous [start, end) ranges of [0, num), one per rank, covering it exactly once.
    With costs (one non-negative value per query) each range gets about 1/world of the
    total cost; otherwise about num / world queries."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if num < 0:
        raise ValueError("num must be >= 0")
    if costs is None:
        bounds = [(num * r) // world for r in range(world + 1)]
    else:
        c = np.asarray(costs, dtype=np.float64)
        if c.shape != (num,):
            raise ValueError("costs must have one value per query")
        if np.any(c < 0) or not np.all(np.isfinite(c)):
            raise ValueError("costs must be finite and non-negative")
        cum = np.concatenate([[0.0], np.cumsum(c)])
        total = cum[-1]
        if total <= 0:
            return shard_ranges(num, world)
        targets = total * np.arange(1, world) / world
        inner = np.searchsorted(cum, targets, side="left").tolist()
        bounds = [0] + [int(min(max(b, 0), num)) for b in inner] + [num]
        for i in range(1, len(bounds)):  # monotone even when costs are zero in stretches
            bounds[i] = max(bounds[i], bounds[i - 1])
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank number over all ranks (no-op without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def broadcast_bytes(data, src: int, device=None):
    """Rank src's uint8 tensor on every rank (its size first, then the bytes, both with the
    process group's broadcast).  `data` is ignored on the other ranks."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank()
    size = torch.zeros(1, dtype=torch.int64, device=device)
    if rank == src:
        size[0] = int(data.numel())
    dist.broadcast(size, src)
    if rank == src:
        buf = data.to(device).contiguous()
    else:
        buf = torch.empty(int(size.item()), dtype=torch.uint8, device=device)
    dist.broadcast(buf, src)
    return buf


def broadcast_tree(ctx, tree, src: int = 0):
    """Replicates rank src's built tree on every rank: src serialises it into one device byte
    buffer (ft_tree_export), the process group broadcasts it (NCCL over NVLink on GPUs) and
    the other ranks import it (ft_tree_import), so the trees are identical everywhere.
    `tree` is rank src's tree; elsewhere a tree to import into (None: a new one).  Returns
    this rank's tree."""
    import torch
    import torch.distributed as dist

    from .hlbvh import import_tree
    dev = f"cuda:{ctx.device}"
    payload = None
    if dist.get_rank() == src:
        payload = torch.empty(tree.export_size(), dtype=torch.uint8, device=dev)
        tree.export(out=payload)
    buf = broadcast_bytes(payload, src, dev)
    if dist.get_rank() == src:
        return tree
    return import_tree(ctx, buf, tree)


def sharded_self_knn(ctx, tree, k: int, rank: int, world: int, costs=None, results=None, result_dists=None,
                     method: int = 1, max_k: int = 32, stream=None):
    """This rank's share of self_knn_query over `tree`: rows for leaf ranks [start, end).
    Returns (start, end, idx, dist); the rows equal those of the full query."""
    import torch

    from .hlbvh import self_knn_query_subset
    start, end = shard_ranges(tree.num_leaves, world, costs)[rank]
    ids = torch.arange(start, end, dtype=torch.int32, device=f"cuda:{ctx.device}")
    idx, dist = self_knn_query_subset(ctx, tree, ids, k, results, result_dists, max_k=max_k, method=method,
                                      stream=stream)
    return start, end, idx, dist
