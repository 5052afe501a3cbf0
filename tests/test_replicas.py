"""Replica plumbing on CPU: world_size-2 gloo ranks (the multi-GPU path shards by instance)."""
import os

import numpy as np
import pytest

from skyrmion_solver_b200.replicas import partition, request_cost
from skyrmion_solver_b200.serving import Request


def _req(rid, arrival, L, C=4):
    p_i = np.array([L, L, L, 2, 3, C, L ** 3, C * L ** 3, 1, 1, 1], np.int32)
    return Request(rid, "nuclear", p_i, np.zeros(8), np.zeros(1), arrival)


def test_partition_is_complete_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    reqs = [_req(k, float(t), int(L)) for k, (t, L) in
            enumerate(zip(np.cumsum(rng.exponential(0.05, 64)), rng.choice([48, 64, 80, 96], 64)))]
    parts = partition(reqs, 4)
    ids = sorted(r.rid for p in parts for r in p)
    assert ids == list(range(64))
    loads = [sum(request_cost(r) for r in p) for p in parts]
    assert max(loads) - min(loads) <= max(request_cost(r) for r in reqs)
    assert [[r.rid for r in p] for p in partition(reqs, 4)] == [[r.rid for r in p] for p in parts]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from skyrmion_solver_b200.replicas import max_over_ranks, sum_over_ranks
        mx = max_over_ranks([1.0 + rank, 10.0 - rank])
        sm = sum_over_ranks([float(rank + 1)])
        reqs = [_req(k, 0.01 * k, 48 + 16 * (k % 3)) for k in range(10)]
        mine = [r.rid for r in partition(reqs, world)[rank]]
        # each rank "serves" its share: converged after 1 + rid seconds, failed for rid 3
        from skyrmion_solver_b200.replicas import gather_objects, merge_served
        rows = [(k, "failed" if k == 3 else "converged", 1.0 + k, 0.01 * k + 1.0 + k) for k in mine]
        merged = merge_served(gather_objects(rows))
        q.put((rank, mx, sm, mine, merged))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_split():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict((r, (mx, sm, mine, merged)) for r, mx, sm, mine, merged in (q.get(timeout=120) for _ in ps))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == [2.0, 10.0]
    assert out[0][1] == out[1][1] == [3.0]
    assert sorted(out[0][2] + out[1][2]) == list(range(10)) and not set(out[0][2]) & set(out[1][2])
    m = out[0][3]
    assert m == out[1][3]                                  # every rank holds the same summary
    assert (m["requests"], m["converged"], m["failed"], m["ranks"]) == (10, 9, 1, 2)
    assert m["wall_s"] == pytest.approx(0.09 + 10.0)       # the latest finish, request 9
    assert m["solves_per_s"] == pytest.approx(9 / 10.09)
    lat = [1.0 + k for k in range(10) if k != 3]
    assert m["p50_s"] == pytest.approx(float(np.percentile(lat, 50)))
    assert sorted(m["requests_per_rank"]) == sorted([len(out[0][2]), len(out[1][2])])
