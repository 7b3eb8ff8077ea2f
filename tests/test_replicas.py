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


def _batch_worker(rank, world, port, out):
    import torch.distributed as dist

    from blockpowerflow_b200 import grid

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        buses, nrhs = grid.batch_sizes(512)
        costs = [replicas.batch_system_cost(1.89 * b, p) for b, p in zip(buses, nrhs)]
        mine = replicas.assign_systems(costs, world)[rank]
        # a stand-in per-system result that names its system: X column sums and the stats
        local = {k: {"x": float(k) * nrhs[k], "niter": 10 + k % 7, "rank": rank} for k in mine}
        merged = replicas.gather_to_root(local)
        tot, mx = replicas.aggregate(sum(nrhs[k] for k in mine), float(len(mine)))
        out.put((rank, sorted(mine), merged, tot, mx))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_shard_the_batch_and_gather_in_order():
    """The batched configuration's 512 systems split over two ranks: every system on exactly one
    rank, the LPT loads balanced, and the one gather returns each system's result under its own
    index on rank 0 (nothing on rank 1), so reassembled results are in the original order."""
    import torch.multiprocessing as mp

    from blockpowerflow_b200 import grid

    buses, nrhs = grid.batch_sizes(512)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    (r0, m0, merged, tot0, mx0), (r1, m1, none1, tot1, mx1) = res
    assert none1 is None
    assert sorted(m0 + m1) == list(range(512)) and not set(m0) & set(m1)
    assert sorted(merged) == list(range(512))
    for k in range(512):
        assert merged[k]["x"] == float(k) * nrhs[k] and merged[k]["niter"] == 10 + k % 7
        assert merged[k]["rank"] == (0 if k in set(m0) else 1)
    assert tot0 == tot1 == sum(nrhs)
    assert mx0 == mx1 == max(len(m0), len(m1))
    costs = [replicas.batch_system_cost(1.89 * b, p) for b, p in zip(buses, nrhs)]
    l0, l1 = sum(costs[k] for k in m0), sum(costs[k] for k in m1)
    assert max(l0, l1) <= 1.05 * (l0 + l1) / 2


def test_batch_system_cost_is_the_sum_over_slices():
    c1 = replicas.batch_system_cost(1000, 16)
    c2 = replicas.batch_system_cost(1000, 64)            # two slices of 32
    assert c2 == pytest.approx(2 * replicas.batch_system_cost(1000, 32))
    assert c1 > 0 and replicas.batch_system_cost(4000, 16) > c1
