"""Sharding independent graphs across ranks (one process per GPU).

Batched diffusion of many independent graphs has no exchange step: each rank
diffuses its own graphs with no collective in the data path. Graphs are
assigned by longest-processing-time first on their cost nnz * F * T (the
gathered bytes of their diffusion): sorted by decreasing cost, each goes to the
least-loaded rank, which keeps the slowest rank within one graph of the mean.
Results can be collected on rank 0 afterwards (``gather_results``) with
``torch.distributed`` (gloo or nccl); that collective is outside the timed
diffusion.

No scl-core counterpart: scl-core runs one process with OpenMP threads.
"""
from __future__ import annotations

import heapq
from typing import Dict, List, Sequence


def lpt_assign(costs: Sequence[float], n_ranks: int) -> List[List[int]]:
    """Graph indices per rank (each list in increasing index order)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    heap = [(0.0, r) for r in range(n_ranks)]
    out: List[List[int]] = [[] for _ in range(n_ranks)]
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def shard_for_rank(costs: Sequence[float], rank: int, world: int) -> List[int]:
    return lpt_assign(costs, world)[rank]


def rank_loads(costs: Sequence[float], assignment: List[List[int]]) -> List[float]:
    return [sum(float(costs[i]) for i in idx) for idx in assignment]


def gather_results(local: Dict[int, "object"], rank: int, world: int, group=None):
    """Collect {graph index: result} from every rank on rank 0 (None elsewhere).
    Results are moved to host memory before the exchange."""
    import torch
    import torch.distributed as dist

    payload = {i: (v.detach().cpu() if isinstance(v, torch.Tensor) else v) for i, v in local.items()}
    if world == 1:
        return payload
    bucket = [None] * world if rank == 0 else None
    dist.gather_object(payload, bucket, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in bucket:
        overlap = set(merged) & set(part)
        if overlap:
            raise RuntimeError(f"graphs {sorted(overlap)} were diffused on more than one rank")
        merged.update(part)
    return merged
