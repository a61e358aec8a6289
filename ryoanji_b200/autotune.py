"""Autotuner of the batched solve: leaf bucket size, target group size, traversal stack depth and target grouping.

Each candidate runs the batched solve on a copy of the caller's bodies (the caller's arrays are not touched) once
to warm up and once timed with CUDA events; the fastest candidate wins. The tuned values change the tree and the
target groups, not the physics: every candidate solves the same systems at the same theta. The grouping is either
fixed windows (tolerance 0, the reference demo's) or the spatial split of each window with tolFactor 2 (the
reference's production grouping), which serves clustered systems with sparse outskirts better.
"""
from __future__ import annotations

import dataclasses
import itertools

import torch

from . import BatchSystem, Context, SolveParams, default_context, solve_batch

DEFAULT_BUCKETS = (16, 32, 64)
DEFAULT_GROUPS = (32, 64)
DEFAULT_STACKS = (512,)  # 1024 entries cost a block per SM and were never faster
DEFAULT_TOLERANCES = (0.0, 2.0)


def tune_batch(systems: list[BatchSystem], bodies: list[torch.Tensor], base: SolveParams | None = None,
               buckets=DEFAULT_BUCKETS, groups=DEFAULT_GROUPS, stacks=DEFAULT_STACKS,
               tolerances=DEFAULT_TOLERANCES, ctx: Context | None = None):
    """@p bodies: x, y, z, m, h (and optionally vx, vy, vz) device tensors of the concatenated systems.
    Returns (best SolveParams, [(bucket, group, stack, tolerance, ms), ...] for every candidate)."""
    ctx = ctx or default_context()
    base = base or SolveParams()
    n = bodies[0].numel()
    work = [b.clone() for b in bodies[:5]]
    out = [torch.empty(n, device=bodies[0].device) for _ in range(4)]
    table = []
    best = None
    for bucket, group, stack, tol in itertools.product(buckets, groups, stacks, tolerances):
        if tol > 0 and group not in (32, 64):
            continue  # spatial groups split windows of 32 or 64
        p = dataclasses.replace(base, bucket_size=bucket, group_size=group, stack_capacity=stack,
                                group_tolerance=tol, timing=False)
        times = []
        for _ in range(2):
            for w, b in zip(work, bodies):
                w.copy_(b)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            solve_batch(systems, *work, *out, params=p, ctx=ctx)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = times[-1]
        table.append((bucket, group, stack, tol, ms))
        if best is None or ms < best[1]:
            best = (p, ms)
    return dataclasses.replace(best[0], timing=base.timing), table
