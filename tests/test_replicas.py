"""Multi-GPU is replicas: the host dispatcher on CPU, world size 2 over gloo.

Wraps are independent, so ranks share the work without a collective on the
data path; these tests run the dispatcher's rank logic as two gloo processes
on 127.0.0.1 with a CPU stand-in for the per-rank solve.
"""

from __future__ import annotations

import os
import socket

import pytest

from nricp_b200.replicas import ReplicaGroup, assign, solve_replicated


def test_assignment_balances_and_covers_every_item_once():
    costs = [5, 1, 1, 1, 1, 1, 9, 2, 2]
    shares = assign(costs, 2)
    assert sorted(shares[0] + shares[1]) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(costs)
    assert all(s == sorted(s) for s in shares)
    assert assign(costs, 2) == shares            # deterministic
    assert assign([1.0], 4) == [[0], [], [], []]


def test_single_process_group_is_the_identity():
    group = ReplicaGroup(backend="gloo")
    assert not group.distributed and group.world == 1
    assert group.max(3.0) == 3.0 and group.sum(2.0) == 2.0
    assert solve_replicated(group, [1, 2, 3], lambda share: [x * 10 for x in share],
                            cost=float) == [10, 20, 30]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    group = ReplicaGroup(backend="gloo", timeout_s=60)
    try:
        cases = [(f"case{i}", float(1 + (i * 7) % 5)) for i in range(11)]
        seen = []

        def solve(share):
            seen.extend(name for name, _ in share)
            return [name.upper() for name, _ in share]

        results = solve_replicated(group, cases, solve, cost=lambda c: c[1])
        group.barrier()
        timing = group.max(1.0 + rank)
        work = group.sum(float(len(seen)))
        queue.put((rank, results, seen, timing, work))
    finally:
        group.close()


def test_two_gloo_ranks_share_the_wraps_and_gather_in_order():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, results, seen, timing, work = queue.get(timeout=120)
        out[rank] = (results, seen, timing, work)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expected = [f"CASE{i}" for i in range(11)]
    assert out[0][0] == expected and out[1][0] is None
    seen0, seen1 = set(out[0][1]), set(out[1][1])
    assert not (seen0 & seen1) and len(seen0 | seen1) == 11   # each wrap solved once
    assert out[0][2] == out[1][2] == 2.0                       # max over ranks
    assert out[0][3] == out[1][3] == 11.0                      # work summed over ranks
