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


def gather_objects(obj, group=None) -> list:
    """`obj` of every rank in rank order, on every rank ([obj] without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out


def merge_served(per_rank) -> dict:
    """Whole-job serving summary from each rank's results, given as lists of
    (rid, status, latency_s, finished_s) with `finished` on the rank's own clock, which
    starts at a common barrier.  Counts add up; the job's wall time is the latest finish
    on any rank; solves/s = converged requests / that wall time; p50 / p99 are over every
    converged request's time-to-converged."""
    import numpy as np
    rows = [r for part in per_rank for r in part]
    lat = np.array([r[2] for r in rows if r[1] == "converged"], dtype=np.float64)
    wall = max((r[3] for r in rows), default=0.0)
    done = int(lat.size)
    return {
        "requests": len(rows),
        "converged": done,
        "failed": sum(r[1] == "failed" for r in rows),
        "not_converged": sum(r[1] == "not_converged" for r in rows),
        "solves_per_s": done / wall if wall > 0 else None,
        "p50_s": float(np.percentile(lat, 50)) if done else None,
        "p99_s": float(np.percentile(lat, 99)) if done else None,
        "wall_s": wall,
        "ranks": len(per_rank),
        "requests_per_rank": [len(p) for p in per_rank],
    }
