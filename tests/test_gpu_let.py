"""The locally essential tree exchange on the GPU (ryo_let_export_f32 and ryoanji_b200/let.py).

- An export against the bounding box of the solve's own bodies holds every cell and body that any of its own target
  groups reaches, so traversing it reproduces the local solve: the same interaction counts and the same forces.
- An export against a far box is a handful of multipoles and no bodies.
- Two ranks on one GPU, exchanging through host memory over gloo (the kernels of the two processes never wait on
  each other), solve one Plummer sphere split into two SFC halves; every body's acceleration agrees with the
  single-GPU solve of the whole sphere to the Barnes-Hut error, against FP64 direct sums.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _arrays(p):
    return [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]


def test_export_for_own_domain_reproduces_the_local_solve():
    import ryoanji_b200 as ryo
    from ryoanji_b200.let import let_export, traverse_export
    p = ds.plummer(1 << 16, seed=61, velocities=False)
    x, y, z, m, h = _arrays(p)
    n = p.n
    out = [torch.zeros(n, device="cuda") for _ in range(4)]
    ctx = ryo.Context(0)
    res = ryo.solve(x, y, z, m, h, *out, params=ryo.SolveParams(theta=0.5), ctx=ctx)
    own = [float(x.min()), float(x.max()), float(y.min()), float(y.max()), float(z.min()), float(z.max())]
    buf, cnt = let_export(own, ctx=ctx)
    assert cnt["numBodies"] > 0 and cnt["numNodes"] <= res.num_nodes
    groups = ryo.solve_arrays(ctx)["groups"].clone()
    again = [torch.zeros(n, device="cuda") for _ in range(4)]
    pot, sp2p, sm2p = traverse_export(buf, cnt, groups, x, y, z, m, h, *again, 1.0, ctx=ctx)
    assert abs(sp2p - res.sum_p2p) <= 1e-3 * res.sum_p2p and abs(sm2p - res.sum_m2p) <= 1e-3 * res.sum_m2p
    a0 = torch.stack(out[1:]).double()
    a1 = torch.stack(again[1:]).double()
    e = (torch.linalg.norm(a1 - a0, dim=0) / torch.linalg.norm(a0, dim=0)).cpu().numpy()
    assert np.percentile(e, 99) <= 1e-6 and e.max() <= 1e-3, (np.percentile(e, 99), e.max())
    assert abs(pot - res.potential_energy) <= 1e-5 * abs(res.potential_energy)


def test_export_for_a_far_box_is_a_few_multipoles():
    import ryoanji_b200 as ryo
    from ryoanji_b200.let import let_export, let_views
    p = ds.uniform_cube(50000, seed=62, eps=0.01)
    x, y, z, m, h = _arrays(p)
    ctx = ryo.Context(0)
    ryo.solve(x, y, z, m, h, *[torch.zeros(p.n, device="cuda") for _ in range(4)], ctx=ctx)
    buf, cnt = let_export([20.0, 21.0, 20.0, 21.0, 20.0, 21.0], ctx=ctx)
    assert cnt["numBodies"] == 0 and cnt["numNodes"] == 9  # the root and its eight children
    v = let_views(buf, cnt)
    assert torch.all(v["childOffsets"][1:] == 0)
    assert abs(float(v["multipoles"][1:, 0].sum()) - float(m.sum())) <= 1e-5 * float(m.sum())


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n, seed, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        import ryoanji_b200 as ryo
        from ryoanji_b200.let import global_box, sfc_partition, solve_distributed
        torch.cuda.set_device(0)
        p = ds.plummer(n, seed=seed, velocities=False)
        # every rank starts with an arbitrary share (every world-th body) ...
        sl = slice(rank, None, world)
        x, y, z, m, h = (torch.from_numpy(np.ascontiguousarray(a[sl])).cuda() for a in (p.x, p.y, p.z, p.m, p.h))
        idx = torch.arange(n, device="cuda", dtype=torch.float32)[sl].contiguous()
        # ... and takes its SFC range of the whole system
        box = global_box(x, y, z)
        x, y, z, m, h, idx = sfc_partition(x, y, z, m, h, box, extra=(idx,))
        k = x.numel()
        acc = [torch.zeros(k, device="cuda") for _ in range(4)]
        order = torch.empty(k, dtype=torch.int32, device="cuda")
        r = solve_distributed(x, y, z, m, h, *acc, params=ryo.SolveParams(theta=0.5), order=order)
        gid = idx[order.long()].long().cpu().numpy()
        out.put((rank, gid, torch.stack(acc[1:]).cpu().numpy(), r.potential_energy, r.exported, r.received))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_two_and_three_ranks_on_one_gpu_match_the_single_solve(world):
    import ryoanji_b200 as ryo
    n, seed = 1 << 17, 63
    p = ds.plummer(n, seed=seed, velocities=False)
    # the single-GPU solve of the whole sphere and the FP64 direct sum on sampled bodies
    x, y, z, m, h = _arrays(p)
    acc = [torch.zeros(n, device="cuda") for _ in range(4)]
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    single = ryo.solve(x, y, z, m, h, *acc, params=ryo.SolveParams(theta=0.5), order=order)
    a_single = np.zeros((3, n))
    a_single[:, order.long().cpu().numpy()] = torch.stack(acc[1:]).cpu().numpy()
    rng = np.random.default_rng(5)
    tgt = np.sort(rng.choice(n, 4096, replace=False))
    orig = _arrays(p)
    _, rx, ry, rz = ryo.direct_targets_f64(torch.from_numpy(tgt).cuda(), *orig)
    ref = torch.stack([rx, ry, rz]).cpu().numpy()
    torch.cuda.synchronize()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, seed, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    parts = [q.get(timeout=600) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    a_dist = np.full((3, n), np.nan)
    energies = set()
    for rank, gid, a, energy, exported, received in parts:
        a_dist[:, gid] = a
        energies.add(round(energy, 12))
        assert sum(e[2] for e in exported) > 0 and sum(r[0] for r in received) > 0
    assert not np.isnan(a_dist).any()  # every body solved once
    assert len(energies) == 1  # the same all-reduced energy on every rank

    def err(a):
        return np.linalg.norm(a[:, tgt] - ref, axis=0) / np.linalg.norm(ref, axis=0)

    e_single, e_dist = err(a_single), err(a_dist)
    assert np.percentile(e_dist, 99) <= max(1.5 * np.percentile(e_single, 99), 1e-3)
    assert e_dist.max() <= max(2.0 * e_single.max(), 5e-3)
    assert abs(energies.pop() - single.potential_energy) <= 2e-4 * abs(single.potential_energy)
