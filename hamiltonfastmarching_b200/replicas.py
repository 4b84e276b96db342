"""Multi-GPU execution by replicas: instances are independent solves, so N GPUs run N processes
(one per GPU, torch.distributed for the plumbing) that each solve their own share of the
instances; there is no collective on the data path. Timing is the max over ranks.

* :func:`assign` splits instances over ranks by estimated work (largest first onto the least
  loaded rank), so that ranks finish together;
* :func:`max_over_ranks` / :func:`sum_over_ranks` reduce a host scalar over the process group
  (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def assign(work: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the instances of each rank: greedy longest-processing-time assignment."""
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    for lst in out:
        lst.sort()
    return out


def _reduce(x: float, op_name: str) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float) -> float:
    return _reduce(x, "MAX")


def sum_over_ranks(x: float) -> float:
    return _reduce(x, "SUM")
