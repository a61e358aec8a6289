"""Placement of systems and requests across ranks (CPU; the multi-rank check runs two gloo processes)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ryoanji_b200 import datasets as ds
from ryoanji_b200.shard import lpt_partition, route_requests, solve_cost


def test_lpt_covers_every_index_once_and_balances():
    sizes, _ = ds.ensemble_sizes(1024, seed=5)
    costs = [solve_cost(int(n)) for n in sizes]
    for ranks in (1, 2, 3, 8):
        parts = lpt_partition(costs, ranks)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: the makespan is within 4/3 of optimal; with many small items it is close to the mean
        assert max(loads) <= 1.02 * np.mean(loads) + max(costs), (ranks, loads)


def test_lpt_edge_cases():
    assert lpt_partition([], 3) == [[], [], []]
    assert lpt_partition([5.0], 2) == [[0], []]
    assert lpt_partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_route_requests_spreads_load():
    reqs = ds.served_requests(200, seed=3, rate_per_s=50.0)
    ranks = route_requests(reqs, 4)
    assert len(ranks) == 200 and set(ranks) <= {0, 1, 2, 3}
    work = np.zeros(4)
    for q, r in zip(reqs, ranks):
        work[r] += solve_cost(q["n"]) * (q["steps"] + 1)
    assert work.max() <= 1.5 * work.mean(), work
    assert route_requests(reqs, 1) == [0] * 200


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes, _ = ds.ensemble_sizes(256, seed=9)
        costs = [solve_cost(int(n)) for n in sizes]
        mine = lpt_partition(costs, world)[rank]  # every rank computes the same placement independently
        t = torch.zeros(len(costs), dtype=torch.int64)
        t[mine] = rank + 1
        dist.all_reduce(t)  # the shares of all ranks must tile the list: each slot set by exactly one rank
        counts = torch.zeros(len(costs), dtype=torch.int64)
        counts[mine] = 1
        dist.all_reduce(counts)
        load = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
        loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(loads, load)
        if rank == 0:
            out.put((counts.tolist(), [float(x) for x in loads], t.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_placement():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    counts, loads, owner = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert counts == [1] * 256
    assert set(owner) == {1, 2}
    assert max(loads) <= 1.05 * (sum(loads) / 2)
