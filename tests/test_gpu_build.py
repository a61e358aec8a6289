"""GPU parity of the build phases against the reference fixtures and the oracle (bit for bit).

SFC keys, sorted order, cornerstone leaves and counts, every linked-octree array and the fixed groups must equal
the reference's; the TreeBuilder drop-in is checked end to end.
"""
import os

import numpy as np
import pytest
import torch

from conftest import golden_cases

pytestmark = pytest.mark.gpu

CASES = golden_cases()
IDS = [os.path.basename(c)[5:-4] for c in CASES]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host_u64(t):
    return t.cpu().numpy().view(np.uint64)


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module", params=CASES, ids=IDS)
def case(request):
    return dict(np.load(request.param))


def box_of(case):
    import ryoanji_b200 as ryo
    return ryo.Box(*[float(v) for v in case["box"]])


def test_keys_bit_exact(case):
    import ryoanji_b200 as ryo
    keys = ryo.compute_sfc_keys(dev(case["x"]), dev(case["y"]), dev(case["z"]), box_of(case))
    assert np.array_equal(host_u64(keys), case["keys"])


def test_keys_double_and_removed_marker(oracle):
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(7)
    n = 50000
    x, y, z = (rng.uniform(-3, 5, n) for _ in range(3))
    box = np.array([-3.0, 5.0, -3.0, 5.0, -3.0, 5.0])
    ref = oracle.sfc_keys(x, y, z, box)
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    keys[::5] = np.int64(-2 ** 63)  # 2^63 as uint64: the removal marker
    out = ryo.compute_sfc_keys(dev(x), dev(y), dev(z), ryo.Box(*box), keys=keys)
    got = host_u64(out)
    marked = np.zeros(n, bool)
    marked[::5] = True
    assert np.all(got[marked] == np.uint64(1 << 63))
    assert np.array_equal(got[~marked], ref[~marked])


@pytest.mark.parametrize("n", [1, 2, 33, 3071, 3072, 3073, 100003])
def test_sort_stable_sizes(n):
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(n)
    k = rng.integers(0, 2 ** 63, n, dtype=np.int64)
    k[rng.integers(0, n, n // 3 + 1)] = k[0]  # duplicates
    keys = dev(k)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ryo.sort_by_key(keys, vals)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(host(keys), k[order])
    assert np.array_equal(host(vals), order.astype(np.int32))


def test_sort_bit_exact(case):
    import ryoanji_b200 as ryo
    keys = dev(case["keys"].view(np.int64))
    vals = torch.arange(len(case["keys"]), dtype=torch.int32, device="cuda")
    ryo.sort_by_key(keys, vals)
    assert np.array_equal(host_u64(keys), case["sorted_keys"])
    assert np.array_equal(host(vals).view(np.uint32), case["order"])


def test_leaves_bit_exact(case):
    import ryoanji_b200 as ryo
    leaves, counts = ryo.compute_octree(dev(case["sorted_keys"].view(np.int64)), int(case["bucket"]))
    assert np.array_equal(host_u64(leaves), case["leaves"])
    assert np.array_equal(host(counts).view(np.uint32), case["counts"])


# buckets that are and are not one less than a power of two: the window maximum over bucket + 1 windows comes from
# power-of-two spans, and 16384 is the largest bucket the leaf construction takes
@pytest.mark.parametrize("kind,bucket", [("plummer", 64), ("halos", 16), ("cube", 1), ("dup", 4), ("tiny", 64),
                                         ("cube", 7), ("halos", 100), ("plummer", 1000), ("big", 16384),
                                         ("edge", 64)])
def test_leaves_against_oracle(oracle, kind, bucket):
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    if kind == "plummer":
        p = ds.plummer(150000, seed=3, velocities=False)
    elif kind == "big":
        p = ds.plummer(120000, seed=8, velocities=False)
    elif kind == "edge":
        p = ds.uniform_cube(65, seed=9)  # one window of bucket + 1 keys
    elif kind == "halos":
        p = ds.hernquist_halos(60000, num_halos=8, seed=4)
    elif kind == "cube":
        p = ds.uniform_cube(5000, seed=5)
    elif kind == "dup":
        p = ds.uniform_cube(4000, seed=6)
        p.x[:] = np.round(p.x * 4) / 4
        p.y[:] = np.round(p.y * 4) / 4
        p.z[:] = np.round(p.z * 4) / 4
    else:
        p = ds.uniform_cube(40, seed=7)
    box = ds.cube_box(p, pad=1e-6)
    keys = oracle.sfc_keys(p.x, p.y, p.z, np.array(box, np.float32))
    sk, _ = oracle.sort_keys(keys)
    l_ref, c_ref = oracle.octree_leaves(sk, bucket)
    leaves, counts = ryo.compute_octree(dev(sk.view(np.int64)), bucket)
    assert np.array_equal(host_u64(leaves), l_ref)
    assert np.array_equal(host(counts).view(np.uint32), c_ref)
    t_ref = oracle.octree_link(l_ref)
    t = ryo.build_octree(leaves)
    for k in ("prefixes", "childOffsets", "parents", "levelRange", "internalToLeaf", "leafToInternal"):
        got = np.asarray(t[k], dtype=np.int32) if k == "levelRange" else host(t[k])
        assert np.array_equal(got.view(t_ref[k].dtype), t_ref[k]), k


def test_link_bit_exact(case):
    import ryoanji_b200 as ryo
    t = ryo.build_octree(dev(case["leaves"].view(np.int64)))
    assert np.array_equal(np.array(t["levelRange"]), case["tree_levelRange"])
    assert np.array_equal(host(t["d_levelRange"]), case["tree_levelRange"])
    for k in ("prefixes", "childOffsets", "parents", "internalToLeaf", "leafToInternal"):
        assert np.array_equal(host(t[k]).view(case["tree_" + k].dtype), case["tree_" + k]), k


def test_fixed_groups(known):
    import ryoanji_b200 as ryo
    g = ryo.compute_fixed_groups(4, 34, 8)
    assert np.array_equal(host(g), known["fixed_groups"])
    g = ryo.compute_fixed_groups(0, 130, 64)
    assert np.array_equal(host(g), [0, 64, 128, 130])


def test_treebuilder_drop_in(case):
    """TreeBuilder::update sorts x, y, z in place and exposes the reference's tree arrays"""
    import ryoanji_b200 as ryo
    x, y, z = dev(case["x"]), dev(case["y"]), dev(case["z"])
    tb = ryo.TreeBuilder(int(case["bucket"]))
    nn = tb.update(x, y, z, box_of(case))
    o = case["order"]
    assert np.array_equal(host(x), case["x"][o]) and np.array_equal(host(z), case["z"][o])
    assert nn == len(case["tree_prefixes"]) and tb.numLeafNodes == len(case["counts"])
    assert tb.maxTreeLevel == 21
    assert np.array_equal(host(tb.order()).view(np.uint32), o)
    assert np.array_equal(host(tb.layout()).view(np.uint32), case["layout"])
    assert np.array_equal(host_u64(tb.nodeKeys()), case["tree_prefixes"])
    assert np.array_equal(host(tb.childOffsets()), case["tree_childOffsets"])
    assert np.array_equal(host(tb.internalToLeaf()), case["tree_internalToLeaf"])
    ni = (len(case["counts"]) - 1) // 7
    assert np.array_equal(host(tb.leafToInternal()), case["tree_leafToInternal"][ni:])
    assert tb.levelRange == list(case["tree_levelRange"])
    # a second update reuses the builder
    nn2 = tb.update(x, y, z, box_of(case))
    assert nn2 == nn


def test_treebuilder_double_coordinates(oracle):
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(12)
    n = 20000
    x, y, z = (rng.normal(0, 0.3, n).clip(-1, 1) for _ in range(3))
    box = np.array([-1.0, 1.0, -1.0, 1.0, -1.0, 1.0])
    keys = oracle.sfc_keys(x, y, z, box)
    sk, order = oracle.sort_keys(keys)
    l_ref, c_ref = oracle.octree_leaves(sk, 32)
    X, Y, Z = dev(x), dev(y), dev(z)
    tb = ryo.TreeBuilder(32)
    tb.update(X, Y, Z, ryo.Box(*box))
    assert np.array_equal(host(X), x[order])
    assert np.array_equal(host_u64(tb.leaves()), l_ref)


def test_bad_box_is_an_error():
    import ryoanji_b200 as ryo
    x = torch.zeros(10, device="cuda")
    with pytest.raises(ryo.RyoError):
        ryo.compute_sfc_keys(x, x, x, ryo.Box(1, 0, 0, 1, 0, 1))
