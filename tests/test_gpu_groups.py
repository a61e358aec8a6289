"""Spatial target groups (cstone::computeGroupSplits) on the GPU.

Group boundaries are integers and must equal, bit for bit, both the oracle's restatement and the reference's own GPU
code (compiled from the reference sources into oracle/_ref when the reference tree was present at build time).
A solve with spatial groups must keep BH accuracy and its per-group interaction counts must equal the oracle's rule
for the same groups.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from conftest import ROOT
from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu

REF_GROUPS = os.path.join(ROOT, "oracle", "_ref", "libryo_ref_groups.so")


def _ref_lib():
    if not os.path.exists(REF_GROUPS):
        pytest.skip("the reference's GPU grouping was not built (no reference tree at build time)")
    lib = C.CDLL(REF_GROUPS)
    lib.ref_group_splits_f32.restype = C.c_long
    return lib


def _tree(p, bucket, oracle):
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    keys = oracle.sfc_keys(p.x, p.y, p.z, box)
    sk, order = oracle.sort_keys(keys)
    leaves, counts = oracle.octree_leaves(sk, bucket)
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    xs, ys, zs, hs = (np.ascontiguousarray(a[order]) for a in (p.x, p.y, p.z, p.h))
    return box, xs, ys, zs, hs, leaves, layout


def _ours(xs, ys, zs, hs, leaves, layout, box, gsize, tol, ratio, use_h=True):
    import ryoanji_b200 as ryo
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    b = ryo.Box(*[float(v) for v in box])
    g = ryo.compute_group_splits(d(xs), d(ys), d(zs), d(hs) if use_h else None, d(leaves.view(np.int64)),
                                 d(layout.view(np.int32)), b, gsize, tol, ratio)
    return g.cpu().numpy().view(np.uint32)


def _reference(xs, ys, zs, hs, leaves, layout, box, gsize, tol):
    lib = _ref_lib()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    X, Y, Z, H = d(xs), d(ys), d(zs), d(hs)
    L, LY = d(leaves.view(np.int64)), d(layout.view(np.int32))
    cap = len(xs) + 2
    out = np.zeros(cap, np.uint32)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    ng = lib.ref_group_splits_f32(C.c_uint32(0), C.c_uint32(len(xs)), p(X), p(Y), p(Z), p(H), p(L),
                                  C.c_int(len(leaves) - 1), p(LY), box.ctypes.data_as(C.c_void_p), C.c_int(gsize),
                                  C.c_float(tol), out.ctypes.data_as(C.c_void_p), C.c_long(cap))
    torch.cuda.synchronize()
    return out[:ng + 1]


CASES = [("plummer", lambda: ds.plummer(60000, seed=1, velocities=False), 64),
         ("cube", lambda: ds.uniform_cube(40000, seed=2, eps=0.002), 32),
         ("halos", lambda: ds.hernquist_halos(50000, num_halos=16, seed=3), 16)]


@pytest.mark.parametrize("name,make,bucket", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("gsize", [32, 64])
def test_groups_match_oracle_bit_for_bit(oracle, name, make, bucket, gsize):
    p = make()
    box, xs, ys, zs, hs, leaves, layout = _tree(p, bucket, oracle)
    for tol, ratio in ((2.0, 8.0), (2.0, 0.0), (0.5, 8.0)):
        want, _ = oracle.group_splits(0, len(xs), xs, ys, zs, hs, leaves, layout, box, gsize, tol, ratio)
        got = _ours(xs, ys, zs, hs, leaves, layout, box, gsize, tol, ratio)
        assert np.array_equal(got, want), (name, gsize, tol, ratio, len(got), len(want))
        assert got[0] == 0 and got[-1] == len(xs) and np.all(np.diff(got.astype(np.int64)) > 0)
        assert np.all(np.diff(got.astype(np.int64)) <= gsize)


@pytest.mark.parametrize("name,make,bucket", CASES, ids=[c[0] for c in CASES])
def test_groups_match_reference_gpu_code(oracle, name, make, bucket):
    p = make()
    box, xs, ys, zs, hs, leaves, layout = _tree(p, bucket, oracle)
    for gsize in (32, 64):
        want = _reference(xs, ys, zs, hs, leaves, layout, box, gsize, 2.0)
        got = _ours(xs, ys, zs, hs, leaves, layout, box, gsize, 2.0, -1.0)
        assert np.array_equal(got, want), (name, gsize, len(got), len(want))


def test_known_answer_case_against_reference_gpu_code(oracle):
    """the reference test's layout (cstone/test/unit_cuda/traversal/groups.cu:170-295) in float"""
    first, last = 4, 128
    lvl1, lvl2 = 1 << 60, 1 << 57
    leaves = np.array([0, lvl1] + [2 * lvl1 + j * lvl2 for j in range(8)] + [k * lvl1 for k in range(3, 8)]
                      + [1 << 63], np.uint64)
    counts = [4, 1, 8, 8, 8, 8, 31, 8, 8, 8, 16, 16, 16, 0, 0]
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    x = np.arange(last, dtype=np.float32)
    y, z = x.copy(), x.copy()
    h = np.full(last, 128.0, np.float32)
    h[first + 64 + 6] = 0.99 * np.sqrt(3.0) / 2
    h[first + 64 + 7] = 1.01 * np.sqrt(3.0) / 2
    for a in (x, y, z):
        a[5] -= 0.01
    box = np.array([0, last, 0, last, 0, last], np.float32)
    tol = float(np.float32(np.sqrt(3.0) / np.cbrt(last ** 3 / 64) * 1.01))
    import ryoanji_b200 as ryo
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got = ryo.compute_group_splits(d(x), d(y), d(z), d(h), d(leaves.view(np.int64)), d(layout.view(np.int32)),
                                   ryo.Box(0, last, 0, last, 0, last), 64, tol, -1.0, first=first, last=last)
    got = got.cpu().numpy().view(np.uint32)
    want, _ = oracle.group_splits(first, last, x, y, z, h, leaves, layout, box, 64, tol, 8.0)
    assert np.array_equal(got, want)
    lib = _ref_lib()
    X, Y, Z, H = d(x), d(y), d(z), d(h)
    L, LY = d(leaves.view(np.int64)), d(layout.view(np.int32))
    out = np.zeros(last + 2, np.uint32)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    ng = lib.ref_group_splits_f32(C.c_uint32(first), C.c_uint32(last), p(X), p(Y), p(Z), p(H), p(L),
                                  C.c_int(len(leaves) - 1), p(LY), box.ctypes.data_as(C.c_void_p), C.c_int(64),
                                  C.c_float(tol), out.ctypes.data_as(C.c_void_p), C.c_long(last + 2))
    assert np.array_equal(got, out[:ng + 1]), (got, out[:ng + 1])


def test_solve_with_spatial_groups(oracle):
    import ryoanji_b200 as ryo
    p = ds.plummer(120000, seed=4, velocities=False)
    res = {}
    for tol in (0.0, 2.0):
        x, y, z, m, h = (torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h))
        n = p.n
        pot, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
        r = ryo.solve(x, y, z, m, h, pot, ax, ay, az, ryo.SolveParams(theta=0.5, group_tolerance=tol))
        tgt = torch.from_numpy(np.random.default_rng(2).choice(n, 2000, replace=False)).cuda()
        _, rx, ry, rz = ryo.direct_targets_f64(tgt, x, y, z, m, h)
        a = torch.stack([ax[tgt], ay[tgt], az[tgt]], 1).double()
        ref = torch.stack([rx, ry, rz], 1)
        err = (torch.linalg.norm(a - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy()
        res[tol] = (r, float(np.percentile(err, 99)))
        if tol > 0:
            arr = ryo.solve_arrays()
            groups = arr["groups"].cpu().numpy().view(np.uint32)
            assert arr["numGroups"] == r.num_groups and len(groups) == r.num_groups + 1
            host = lambda t: np.ascontiguousarray(t.cpu().numpy())  # noqa: E731
            xs, ys, zs, ms, hs = (host(t) for t in (x, y, z, m, h))
            m2p, p2p, _ = oracle.traverse_rule(groups[:-1], groups[1:], xs, ys, zs, hs, ms,
                                               dict(childOffsets=host(arr["childOffsets"]),
                                                    internalToLeaf=host(arr["internalToLeaf"])),
                                               host(arr["layout"]).view(np.uint32), host(arr["centers"]),
                                               host(arr["multipoles"]))
            assert np.array_equal(arr["groupM2P"].cpu().numpy().view(np.uint32), m2p)
            assert np.array_equal(arr["groupP2P"].cpu().numpy().view(np.uint32), p2p)
    assert res[2.0][1] < 2.5e-3, res[2.0][1]
    assert res[2.0][0].num_groups >= res[0.0][0].num_groups
