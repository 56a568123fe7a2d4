"""One process per GPU: independent LPs per rank, no collective on the data path.

The single-LP inner solve does not shard (its PCG is one dependency chain per
Newton step), so multi-GPU runs are replicas: each rank solves its own LPs.
Two helpers:

* :func:`partition_by_nnz` — deterministic longest-processing-time split of
  a batch of LPs across ranks by nonzero count (the work proxy of H·p and of
  the preconditioner);
* :func:`max_over_ranks` — the job time of a step is the slowest rank's
  time (all-reduce MAX; NCCL with CUDA tensors, gloo on CPU).
"""

from __future__ import annotations

import heapq
from typing import List, Sequence


def partition_by_nnz(nnz: Sequence[int], world: int) -> List[List[int]]:
    """Indices of `nnz` per rank, heaviest first onto the least-loaded rank."""
    if world < 1:
        raise ValueError("world must be positive")
    order = sorted(range(len(nnz)), key=lambda i: (-int(nnz[i]), i))
    heap = [(0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(nnz[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float) -> float:
    """Maximum of `value` over the ranks of the default process group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
