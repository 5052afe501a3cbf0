"""Multi-GPU plumbing for independent solves (one process and one engine per GPU).

Solves never exchange data: a lattice of up to 192^3 sites fits one B200 many
times over, so several GPUs serve disjoint sets of instances and the only
cross-rank traffic is control: timings reduced to their maximum over ranks
(the job is as slow as its slowest GPU) and a deterministic split of a
request stream.  Both run over ``torch.distributed`` (NCCL on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations

import heapq


def max_over_ranks(values, group=None, device=None):
    """Element-wise maximum of a list of floats over all ranks (returns a list of floats)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(v) for v in t.cpu()]


def sum_over_ranks(values, group=None, device=None):
    """Element-wise sum of a list of floats over all ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [float(v) for v in t.cpu()]


def request_cost(req) -> int:
    """Work estimate of a relaxation request: field values (components x sites)."""
    p_i = req.p_i
    return int(p_i[5]) * int(p_i[6])


def partition(requests, world: int):
    """Split requests over `world` ranks: in arrival order, each goes to the rank with the
    least work assigned so far (ties to the lowest rank).  Deterministic, so every rank
    computes the same split without communicating.  Returns one list per rank."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for req in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        load, r = heapq.heappop(heap)
        out[r].append(req)
        heapq.heappush(heap, (load + request_cost(req), r))
    return out
