"""Multi-rank host path on CPU (gloo, world_size 2): system assignment and the end-of-run
aggregation bench.py uses for N > 1 (sum of converged RHS, max of the per-rank times)."""
import os
import socket

import pytest

from blockpowerflow_b200 import replicas


def test_lpt_assignment_balances_and_covers():
    costs = [replicas.solve_cost(n, 7 * n, p) for n, p in
             [(530, 16), (16998, 64), (2000, 8), (5000, 32), (300, 64), (9000, 16), (1200, 40)]]
    for world in (1, 2, 3, 4):
        parts = replicas.assign_systems(costs, world)
        assert sorted(i for part in parts for i in part) == list(range(len(costs)))
        loads = [sum(costs[i] for i in part) for part in parts]
        # LPT bound: max load <= (4/3 - 1/(3 world)) * optimum <= 4/3 * max(mean, largest)
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) + 1e-6
    assert replicas.assign_systems([1.0, 1.0], 2) == [[0], [1]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [5.0, 3.0, 3.0, 2.0, 1.0]
        mine = replicas.assign_systems(costs, world)[rank]
        rhs = 64.0 * len(mine)            # every system converged with 64 RHS
        ms = 10.0 * (rank + 1)            # rank 1 is the slower one
        tot, mx = replicas.aggregate(rhs, ms)
        out.put((rank, mine, tot, mx))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_aggregate():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=120) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    res.sort()
    assert res[0][2] == res[1][2] == 64.0 * 5       # all systems counted once
    assert res[0][3] == res[1][3] == 20.0            # max over ranks
    assert sorted(res[0][1] + res[1][1]) == [0, 1, 2, 3, 4]
