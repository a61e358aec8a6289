"""One system spread over several GPUs: the locally essential tree (LET) exchange.

The reference spreads one large system over MPI ranks with cstone's focused octrees: every rank keeps its own SFC
range of bodies and receives, from every other rank, the multipoles and bodies of that rank's tree that its own
targets need (cstone/include/cstone/focus/octree_focus_mpi.hpp:629, globalExchange, and the peer exchange it feeds).
Here one process drives one GPU, torch.distributed carries the exchange (NCCL on GPUs, or gloo through host memory),
and each step is a call of the library:

1. the global box: an all-reduce of the ranks' coordinate bounds (one cube over all bodies, so the SFC keys and the
   node geometry agree between ranks);
2. the local solve of the rank's own bodies in that box (ryo_solve_f32: sort, tree, upsweep, traversal), which sorts
   the bodies in place, as the single-GPU solve does;
3. the bounding boxes of every rank's bodies, all-gathered;
4. for every other rank, the export of this rank's tree against that rank's box (ryo_let_export_f32);
5. an all-to-all of the exports (sizes first, then one packed buffer per pair);
6. the traversal of every received tree by the rank's own target groups (ryo_traverse_f32), accumulated into the
   same outputs;
7. the total potential energy, all-reduced.

Every rank takes the same collective steps in the same order. Accelerations agree with a single-GPU solve of the
whole system to the Barnes-Hut error: each rank's tree is built from its own bodies, so cells near the domain
boundaries group bodies differently than one tree of all bodies would. `sfc_partition` gives each rank a contiguous
SFC range of the bodies it holds, the decomposition this exchange is designed for.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _abi, lib
from . import (Box, Context, SolveParams, _check, _ptr, _same_device, _stream, compute_sfc_keys, default_context,
               solve, solve_arrays, traverse)

_FIELDS = ("numNodes", "numLeaves", "numBodies", "words")


@dataclasses.dataclass
class DistributedSolve:
    """result of solve_distributed on one rank"""
    box: tuple                 # the global cube (xmin, xmax, ymin, ymax, zmin, zmax)
    local: object              # SolveStats of the local solve (own tree only)
    potential_energy: float    # 0.5 G sum m phi over all bodies of all ranks
    exported: list             # per rank: (nodes, leaves with bodies, bodies) sent to it (zeros for self)
    received: list             # per rank: (nodes, leaves with bodies, bodies) received from it
    remote_p2p: int            # bodies summed directly from received trees, over this rank's targets
    remote_m2p: int            # cells approximated from received trees, over this rank's targets


def _coll_device(group):
    """collectives of gloo run on host tensors, of NCCL on the current GPU"""
    import torch.distributed as dist
    return torch.device("cpu") if dist.get_backend(group) == "gloo" else torch.device("cuda",
                                                                                       torch.cuda.current_device())


def global_box(x, y, z, group=None, pad: float = 1e-6) -> tuple:
    """the cube over the bodies of every rank: lower corner at the minimum, side the largest extent (padded)"""
    import torch.distributed as dist
    dev = _coll_device(group)
    if x.numel() > 0:
        lo = torch.stack([x.min(), y.min(), z.min()]).double().to(dev)
        hi = torch.stack([x.max(), y.max(), z.max()]).double().to(dev)
    else:
        lo = torch.full((3,), float("inf"), dtype=torch.float64, device=dev)
        hi = torch.full((3,), -float("inf"), dtype=torch.float64, device=dev)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    lo, hi = lo.cpu().numpy(), hi.cpu().numpy()
    ext = float((hi - lo).max()) * (1 + pad)
    ext = ext if ext > 0 else 1.0
    return (float(lo[0]), float(lo[0]) + ext, float(lo[1]), float(lo[1]) + ext, float(lo[2]), float(lo[2]) + ext)


def exchange(send: list, group=None) -> list:
    """all-to-all of one int32 tensor per destination rank (None or empty for none); returns one per source rank"""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = _coll_device(group)
    sizes = torch.tensor([0 if t is None else t.numel() for t in send], dtype=torch.int64, device=dev)
    got = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(got, sizes, group=group)
    got_l, sizes_l = got.cpu().tolist(), sizes.cpu().tolist()
    parts = [t.reshape(-1).to(dev) for t in send if t is not None and t.numel() > 0]
    flat = torch.cat(parts) if parts else torch.empty(0, dtype=torch.int32, device=dev)
    out = torch.empty(sum(got_l), dtype=torch.int32, device=dev)
    dist.all_to_all_single(out, flat, output_split_sizes=got_l, input_split_sizes=sizes_l, group=group)
    res, o = [], 0
    for k in got_l:
        res.append(out[o:o + k])
        o += k
    return res


def let_export(peer_box, ctx: Context | None = None, stream=None) -> tuple[torch.Tensor, dict]:
    """ryo_let_export_f32: the packed export of the last solve's tree for a box (xmin, xmax, ymin, ymax, zmin, zmax);
    (int32 device tensor of counts['words'] words, counts)"""
    ctx = ctx or default_context()
    b = (C.c_float * 6)(*[float(v) for v in peer_box])
    cnt = _abi.LetCounts()
    st = lib.ryo_let_export_f32(ctx.handle, b, None, 0, C.byref(cnt), _stream(stream, ctx))
    if st != _abi.ERR_CAPACITY:
        _check(st, ctx)
    buf = torch.empty(max(1, int(cnt.words)), dtype=torch.int32, device=torch.device("cuda", ctx.device))
    _check(lib.ryo_let_export_f32(ctx.handle, b, C.c_void_p(buf.data_ptr()), C.c_size_t(buf.numel()), C.byref(cnt),
                                  _stream(stream, ctx)), ctx)
    return buf[:int(cnt.words)], {k: int(getattr(cnt, k)) for k in _FIELDS}


def let_views(buf: torch.Tensor, counts: dict) -> dict:
    """typed views of a packed export (the layout of ryo_let_export_f32)"""
    N, L, B = counts["numNodes"], counts["numLeaves"], counts["numBodies"]
    f = buf.view(torch.float32)
    o = 14 * N + L + 2
    return dict(centers=f[:4 * N].view(N, 4), multipoles=f[4 * N:12 * N].view(N, 8),
                childOffsets=buf[12 * N:13 * N], internalToLeaf=buf[13 * N:14 * N], layout=buf[14 * N:o],
                x=f[o:o + B], y=f[o + B:o + 2 * B], z=f[o + 2 * B:o + 3 * B], m=f[o + 3 * B:o + 4 * B],
                h=f[o + 4 * B:o + 5 * B], numNodes=N)


def traverse_export(buf, counts, groups, x, y, z, m, h, p, ax, ay, az, G: float, ctx: Context | None = None,
                    stream=None):
    """the field of a received export at this rank's sorted bodies (targets grouped by @p groups), added to p, ax,
    ay, az; returns (0.5 G sum m phi, sumP2P, sumM2P)"""
    import ryoanji_b200 as ryo
    v = let_views(buf, counts)
    # an export without bodies still passes valid source pointers: they are never read
    src = [v[k] if counts["numBodies"] > 0 else buf.view(torch.float32)[:1] for k in ("x", "y", "z", "m", "h")]
    init = 1 if v["numNodes"] > 1 else 0
    pot = traverse(groups, init, x, y, z, m, h, *src, v["childOffsets"], v["internalToLeaf"], v["layout"],
                   v["centers"], v["multipoles"], G, 0, None, p, ax, ay, az, ctx=ctx, stream=stream)
    st = ryo.read_bh_stats(ctx)
    return pot, st[0], st[2]


def sfc_partition(x, y, z, m, h, box: tuple, group=None, bits: int = 15, extra=()):
    """this rank's share of a system whose bodies are spread over the ranks in any way: every rank gets a contiguous
    range of the Hilbert curve of @p box with about the same number of bodies. A histogram of the top @p bits key
    bits is all-reduced, cut into equal shares, and the bodies are exchanged all-to-all. Returns the rank's new
    (x, y, z, m, h, *extra) float32 device tensors (arrays of @p extra travel with the bodies)."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    dev = x.device
    keys = compute_sfc_keys(x, y, z, Box(*box))
    top = (keys >> (63 - bits)).to(torch.int64)
    hist = torch.bincount(top, minlength=1 << bits).to(torch.int64)
    cdev = _coll_device(group)
    hist_c = hist.to(cdev)
    dist.all_reduce(hist_c, group=group)
    cum = torch.cumsum(hist_c.cpu(), 0).numpy()
    total = int(cum[-1]) if len(cum) else 0
    # bucket b goes to the rank that holds the body count before it: equal shares along the curve
    before = np.concatenate([[0], cum[:-1]])
    owner = np.minimum((before * world) // max(total, 1), world - 1).astype(np.int64)
    dest = torch.from_numpy(owner).to(dev)[top]
    order = torch.argsort(dest, stable=True)
    counts = torch.bincount(dest, minlength=world)
    cols = [x, y, z, m, h, *extra]
    packed = torch.stack([c[order].float() for c in cols], 1)  # bodies x columns, grouped by destination
    send_sizes = (counts * len(cols)).to(torch.int64)
    got = torch.empty(world, dtype=torch.int64, device=cdev)
    dist.all_to_all_single(got, send_sizes.to(cdev), group=group)
    out = torch.empty(int(got.sum()), dtype=torch.float32, device=cdev)
    dist.all_to_all_single(out, packed.reshape(-1).to(cdev), output_split_sizes=got.cpu().tolist(),
                           input_split_sizes=send_sizes.cpu().tolist(), group=group)
    mine = out.to(dev).view(-1, len(cols))
    return tuple(mine[:, k].contiguous() for k in range(len(cols)))


def solve_distributed(x, y, z, m, h, p, ax, ay, az, params: SolveParams | None = None, group=None,
                      ctx: Context | None = None, stream=None, order=None) -> DistributedSolve:
    """Barnes-Hut forces of one system whose bodies are spread over the ranks of @p group, this rank holding x, y, z,
    m, h (float32, on its GPU; an SFC range from sfc_partition is the intended share). Sorts this rank's bodies in
    place along the curve of the global box and overwrites p, ax, ay, az with the field of every rank's bodies, as
    ryo_solve_f32 does for one GPU; @p order (int32, optional) receives the sorted bodies' indices in the rank's input
    order. Open boundaries, quadrupole expansions."""
    import torch.distributed as dist
    ctx = ctx or default_context()
    _same_device(ctx, x, y, z, m, h, p, ax, ay, az)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    params = params or SolveParams()
    box = global_box(x, y, z, group)
    local = solve(x, y, z, m, h, p, ax, ay, az,
                  params=dataclasses.replace(params, box=Box(*box), timing=False), order=order, ctx=ctx,
                  stream=stream)
    cdev = _coll_device(group)
    mine = torch.tensor([float(x.min()), float(x.max()), float(y.min()), float(y.max()), float(z.min()),
                         float(z.max())], dtype=torch.float32, device=cdev)
    boxes = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(boxes, mine, group=group)
    send, exported = [None] * world, [(0, 0, 0)] * world
    meta = torch.zeros(world, 4, dtype=torch.int64)
    for q in range(world):
        if q == rank:
            continue
        buf, cnt = let_export(boxes[q].cpu().tolist(), ctx=ctx, stream=stream)
        send[q] = buf
        exported[q] = (cnt["numNodes"], cnt["numLeaves"], cnt["numBodies"])
        meta[q] = torch.tensor([cnt[k] for k in _FIELDS])
    got_meta = torch.empty_like(meta).to(cdev)
    dist.all_to_all_single(got_meta, meta.to(cdev), group=group)
    got_meta = got_meta.cpu()
    recv = exchange(send, group)
    groups = solve_arrays(ctx)["groups"].clone()
    pot_remote, rp2p, rm2p = 0.0, 0, 0
    received = [(0, 0, 0)] * world
    dev = torch.device("cuda", ctx.device)
    for q in range(world):
        if q == rank:
            continue
        cnt = dict(zip(_FIELDS, got_meta[q].tolist()))
        received[q] = (cnt["numNodes"], cnt["numLeaves"], cnt["numBodies"])
        buf = recv[q].to(dev)
        pr, s2, s3 = traverse_export(buf, cnt, groups, x, y, z, m, h, p, ax, ay, az, params.G, ctx=ctx,
                                     stream=stream)
        pot_remote += pr
        rp2p += s2
        rm2p += s3
    energy = torch.tensor([local.potential_energy + pot_remote], dtype=torch.float64, device=cdev)
    dist.all_reduce(energy, group=group)
    return DistributedSolve(box=box, local=local, potential_energy=float(energy.item()), exported=exported,
                            received=received, remote_p2p=int(rp2p), remote_m2p=int(rm2p))
