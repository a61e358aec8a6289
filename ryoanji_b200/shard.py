"""Placement of independent systems and requests on the GPUs of one node (one process per GPU).

Batched systems and served requests do not interact, so several GPUs split them with no device-side exchange: every
rank computes the same placement from the same list and solves its own share. Costs are estimated as N log2 N per
solve (tree build and traversal both grow that way), times the number of solves for a request.

- lpt_partition: longest-processing-time-first placement of a known list (the batched ensemble);
- route_requests: online placement in arrival order onto the rank with the least estimated outstanding work (the
  served stream; a request's work is charged to its rank from its arrival until its estimated completion).
"""
from __future__ import annotations

import heapq
import math


def solve_cost(n: int) -> float:
    return float(n) * math.log2(max(int(n), 2))


def lpt_partition(costs, num_ranks: int) -> list[list[int]]:
    """indices of @p costs for every rank: largest first, each onto the least-loaded rank (ties: lowest rank)"""
    if num_ranks < 1:
        raise ValueError("num_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(num_ranks)]
    parts: list[list[int]] = [[] for _ in range(num_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for p in parts:
        p.sort()
    return parts


def route_requests(requests, num_ranks: int, rate: float = 2.0e8) -> list[int]:
    """rank of every request (dicts with 'arrival' seconds, 'n' bodies and 'steps'), in arrival order: the rank whose
    estimated backlog at the arrival time is smallest; @p rate is the assumed throughput in cost units per second"""
    if num_ranks < 1:
        raise ValueError("num_ranks must be >= 1")
    busy_until = [0.0] * num_ranks
    ranks = []
    for q in requests:
        t = q["arrival"]
        backlog = [max(0.0, b - t) for b in busy_until]
        r = min(range(num_ranks), key=lambda k: (backlog[k], k))
        work = solve_cost(q["n"]) * (q["steps"] + 1) / rate
        busy_until[r] = max(busy_until[r], t) + work
        ranks.append(r)
    return ranks
