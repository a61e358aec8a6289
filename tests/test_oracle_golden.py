"""The CPU oracle against the reference's own outputs (golden fixtures written by tests/golden/make_golden.py).

Integer outputs are compared bit for bit; the float upsweep too (same operation order); the CPU tree walk,
direct sum and Ewald to round-off.
"""
import os

import numpy as np
import pytest

from conftest import golden_cases

CASES = golden_cases()


@pytest.fixture(scope="module", params=CASES, ids=[os.path.basename(c)[5:-4] for c in CASES])
def case(request):
    return dict(np.load(request.param))


def test_keys(oracle, case):
    keys = oracle.sfc_keys(case["x"], case["y"], case["z"], case["box"])
    assert np.array_equal(keys, case["keys"])
    assert np.array_equal(oracle.box_dim_bits(case["box"]), case["bits"])


def test_sort(oracle, case):
    sk, order = oracle.sort_keys(case["keys"])
    assert np.array_equal(sk, case["sorted_keys"])
    assert np.array_equal(order, case["order"])


def test_leaves(oracle, case):
    leaves, counts = oracle.octree_leaves(case["sorted_keys"], int(case["bucket"]))
    assert np.array_equal(leaves, case["leaves"])
    assert np.array_equal(counts, case["counts"])


def test_link(oracle, case):
    t = oracle.octree_link(case["leaves"])
    for k in ("prefixes", "childOffsets", "parents", "levelRange", "internalToLeaf", "leafToInternal"):
        assert np.array_equal(t[k], case["tree_" + k]), k


def _sorted(case):
    o = case["order"]
    return [case[k][o] for k in ("x", "y", "z", "m", "h")]


def _tree(oracle, case):
    return oracle.octree_link(case["leaves"])


def test_upsweep_float_order_is_bit_exact(oracle, case):
    xs, ys, zs, ms, hs = _sorted(case)
    t = _tree(oracle, case)
    centers, mp = oracle.upsweep(xs, ys, zs, ms, case["layout"], t, float(case["theta"]), case["box"], mode=0)
    assert np.array_equal(centers, case["centers"])
    assert np.array_equal(mp, case["multipoles"])


def test_upsweep_double_close_to_reference(oracle, case):
    xs, ys, zs, ms, hs = _sorted(case)
    t = _tree(oracle, case)
    c1, m1 = oracle.upsweep(xs, ys, zs, ms, case["layout"], t, float(case["theta"]), case["box"], mode=1)
    c0 = case["centers"]
    scale = np.abs(c0[:, :3]).max()
    assert np.abs(c1[:, :3] - c0[:, :3]).max() <= 2e-6 * scale
    m0 = case["multipoles"]
    assert np.allclose(m1[:, 0], m0[:, 0], rtol=1e-5, atol=0)


def test_gravity_cpu(oracle, case):
    if "grav_ax" not in case:
        pytest.skip("no CPU walk for this case")
    xs, ys, zs, ms, hs = _sorted(case)
    t = _tree(oracle, case)
    u, pot, ax, ay, az = oracle.gravity_cpu(t, case["centers"], case["multipoles"], case["layout"], xs, ys, zs, hs, ms,
                                            case["box"])
    for a, k in ((ax, "grav_ax"), (ay, "grav_ay"), (az, "grav_az"), (pot, "grav_pot")):
        assert np.array_equal(a, case[k]), k
    assert abs(u - float(case["grav_u"])) <= 1e-5 * abs(float(case["grav_u"]))


def test_direct_sum(oracle, case):
    if "direct_ax" not in case:
        pytest.skip("no direct sum for this case")
    x, y, z, m, h = _sorted(case)
    idx = np.arange(0, len(x), 7)
    pot, ax, ay, az = oracle.direct(x, y, z, h, m, idx, G=1.0)
    for a, k in ((pot, "direct_pot"), (ax, "direct_ax"), (ay, "direct_ay"), (az, "direct_az")):
        ref = case[k][idx]
        assert np.allclose(a, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), k


def test_ewald(oracle, case):
    if "ewald_ax" not in case:
        pytest.skip("not periodic")
    xs, ys, zs, ms, hs = (a.astype(np.float64) for a in _sorted(case))
    rc = case["centers"][0, :3].astype(np.float64)
    mr = case["multipoles"][0].astype(np.float64)
    u, pot, ax, ay, az = oracle.ewald(rc, mr, xs, ys, zs, ms, case["box"].astype(np.float64), G=1.0)
    for a, k in ((ax, "ewald_ax"), (ay, "ewald_ay"), (az, "ewald_az"), (pot, "ewald_pot")):
        assert np.allclose(a, case[k], rtol=1e-12, atol=1e-12 * np.abs(case[k]).max()), k
    assert abs(u - float(case["ewald_u"])) <= 1e-12 * abs(float(case["ewald_u"]))


def test_known_answers(oracle, known):
    h1, h2 = known["p2p_h"]
    for h, ref in ((h1, known["p2p_base"]), (h2, known["p2p_soft"])):
        a = oracle.p2p([1, 1, 1], [2, 2, 2], 1.0, h, h)
        a = oracle.p2p([1, 1, 1], [-2, -2, -2], 1.0, h, h, a)
        assert np.allclose(a, ref, rtol=0, atol=1e-10)
    # self interaction is exactly zero for non-zero softening (ryoanji/test/nbody/kernel.cpp:68-78)
    assert np.array_equal(oracle.p2p([0, 0, 0], [0, 0, 0], 1.0, 0.1, 0.1), np.zeros(4))
    e1 = oracle.ewald_single_particle_energy(1.0, 1, 1.0)
    e2 = oracle.ewald_single_particle_energy(1.0, 1, 2.0)
    assert abs(e1 - known["ewald_single"][0]) < 1e-10 and abs(e2 - known["ewald_single"][1]) < 1e-10


def test_m2p_matches_p2p_far_away(oracle):
    """the cartesian quadrupole reproduces the direct sum of its sources far away (cartesian_qpole.cpp:27-76)"""
    rng = np.random.default_rng(11)
    x, y, z = (rng.uniform(-1, 1, 100) for _ in range(3))
    m = rng.uniform(0, 1, 100)
    c, q = oracle.p2m(x, y, z, m)
    target = np.array([-8.0, 0.0, 0.0])
    ref = np.zeros(4)
    for s in range(100):
        ref = oracle.p2p(target, [x[s], y[s], z[s]], m[s], 0.0, 0.0, ref)
    approx = oracle.m2p(target, c[:3], q)
    assert np.abs(approx - ref).max() < 1e-3


def test_mixed_dimension_cell_contains_point(oracle):
    """the fork's cell index puts every point inside its key's cell for fitted boxes (sfc.cpp:69-100)"""
    box = np.array([-0.0011882485223581088, 0.0011884225944410061, -0.0011882157500425073, 0.001188368630643466,
                    -0.012426126792806139, 0.045320500145225831])
    bits = None
    import ctypes as C
    rng = np.random.default_rng(42)
    n = 20000
    x = rng.uniform(box[0], box[1], n)
    y = rng.uniform(box[2], box[3], n)
    z = rng.uniform(box[4], box[5], n)
    x[0], y[0], z[0] = -2.3742214883045176e-05, 9.6842915978489733e-08, 0.010289945748438454
    keys = oracle.sfc_keys(x, y, z, box)
    b = (C.c_uint * 3)()
    oracle.lib.orc_box_dim_bits_f64(box.ctypes.data_as(C.c_void_p), b)
    bits = list(b)
    assert bits[0] == 16 and bits[2] == 21
    L = box[1::2] - box[0::2]
    outside = 0
    for i in range(0, n, 37):
        ib = oracle.hilbert_ibox(int(keys[i]), 21, bits)
        half = [0.5 / 2 ** 21 * L[d] * 2 ** (21 - bits[d]) for d in range(3)]
        c = [box[2 * d] + (ib[2 * d + 1] + ib[2 * d]) * half[d] for d in range(3)]
        s = [(ib[2 * d + 1] - ib[2 * d]) * half[d] for d in range(3)]
        p = (x[i], y[i], z[i])
        tol = 1e-12 * L.max()
        outside += any(abs(p[d] - c[d]) > s[d] + tol for d in range(3))
    assert outside == 0


def test_reference_wrapper_agrees_when_present(oracle):
    """if the reference compiled here, the restatement equals it on a fresh random case (not only the fixtures)"""
    from pyoracle import Oracle, have_reference
    if not have_reference():
        pytest.skip("reference not built here")
    ref = Oracle(reference=True)
    rng = np.random.default_rng(99)
    n = 3000
    x, y, z = (rng.standard_normal(n).astype(np.float32) * 0.2 for _ in range(3))
    box = np.array([-2, 2, -1.5, 1.5, -1, 1], np.float32)
    k1, k2 = oracle.sfc_keys(x, y, z, box), ref.sfc_keys(x, y, z, box)
    assert np.array_equal(k1, k2)
    s1, _ = oracle.sort_keys(k1)
    l1, c1 = oracle.octree_leaves(s1, 12)
    l2, c2 = ref.octree_leaves(s1, 12)
    assert np.array_equal(l1, l2) and np.array_equal(c1, c2)


# ---------------------------------------------------------------------------------------------------------------
# spatial target groups: the reference's own known answers (cstone/test/unit_cuda/traversal/groups.cu:58-295)

def _octree_divide_divide2():
    """the leaf keys of OctreeMaker{}.divide().divide(2): root split into eight, then node 2 split into eight"""
    lvl1 = 1 << 60
    lvl2 = 1 << 57
    keys = [0, lvl1] + [2 * lvl1 + j * lvl2 for j in range(8)] + [k * lvl1 for k in range(3, 8)] + [1 << 63]
    return np.array(keys, np.uint64)


def test_group_find_splits_known_answer():
    orc = __import__("pyoracle").Oracle(reference=False)
    n = 64
    pos = np.zeros((n, 4))
    for i in range(n):
        pos[i] = [i, i, i, n]
    pos[0] = [-1, -1, -1, n]                # split at 0 (distance)
    pos[2, 3] = 0.99 * np.sqrt(3.0)         # split at 2 (interaction radius)
    pos[31, :3] -= 0.5                      # split at 31
    pos[33, :3] -= 0.5                      # split at 33
    mask = orc.find_splits(pos, 3.01)
    assert [b for b in range(64) if (mask >> b) & 1] == [0, 2, 31, 33]


@pytest.mark.parametrize("a,b,want", [
    (0, 0, [64]), (1, 0, [1, 63]), (0, 1 << 30, [63, 1]), (2, 0, [2, 62]), (3, 0, [1, 1, 62]),
    (1 << 31, 1, [32, 1, 31]), (0, 8, [36, 28])])
def test_group_make_splits_known_answers(a, b, want):
    orc = __import__("pyoracle").Oracle(reference=False)
    assert list(orc.make_splits(a | (b << 32))) == want


def test_group_make_splits_dense_masks():
    orc = __import__("pyoracle").Oracle(reference=False)
    got = list(orc.make_splits(0xFFFFFFFF | (0x6FFFFFFF << 32)))
    assert got[:63] == [2 if i == 60 else 1 for i in range(63)]
    got = list(orc.make_splits(0xFFFFFFFF | (0x7FFFFFFF << 32)))
    assert got[:63] == [1] * 63


def _group_volumes_case():
    first, last, gsize = 4, 128, 64
    leaves = _octree_divide_divide2()
    counts = [4, 1, 8, 8, 8, 8, 31, 8, 8, 8, 16, 16, 16, 0, 0]
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    x = np.arange(last, dtype=np.float64)
    y, z = x.copy(), x.copy()
    h = np.full(last, 128.0)
    h[first + gsize + 6] = 0.99 * np.sqrt(3.0) / 2
    h[first + gsize + 7] = 1.01 * np.sqrt(3.0) / 2
    x[5] -= 0.01
    y[5] -= 0.01
    z[5] -= 0.01
    box = np.array([0, last, 0, last, 0, last], np.float64)
    dist_crit = np.cbrt(box[1] ** 3 / 64)
    return first, last, x, y, z, h, leaves, layout, box, dist_crit


def test_group_volumes_known_answers():
    orc = __import__("pyoracle").Oracle(reference=False)
    first, last, x, y, z, h, leaves, layout, box, dist_crit = _group_volumes_case()
    tol = float(np.float32(np.sqrt(3.0) / dist_crit * 1.01))
    _, counts = orc.group_splits(first, last, x, y, z, h, leaves, layout, box, 64, tol, 0.0)
    assert list(counts) == [2, 2]
    tol = float(np.float32(np.sqrt(3.0) / dist_crit * 0.99))
    _, counts = orc.group_splits(first, last, x, y, z, h, leaves, layout, box, 64, tol, 0.0)
    assert list(counts) == [64, 60]
    # fixed groups (4, 68, 128) split into (4, 6, 68, 75, 128): by distance after body 5, by interaction radius after
    # body 74 (the window-extent criterion, which this layout would also trigger, is off here; its behaviour is
    # pinned against the reference's compiled GPU code in tests/test_gpu_groups.py)
    tol = float(np.float32(np.sqrt(3.0) / dist_crit * 1.01))
    groups, _ = orc.group_splits(first, last, x, y, z, h, leaves, layout, box, 64, tol, 0.0)
    assert list(groups) == [4, 6, 68, 75, 128]


# ---------------------------------------------------------------------------------------------------------------
# monopole + dipole + quadrupole expansions: restatement against the reference's own code (signed masses)

@pytest.fixture(scope="module")
def ref_oracle():
    import pyoracle
    if not pyoracle.have_reference():
        pytest.skip("reference wrapper not built")
    return pyoracle.Oracle(reference=True)


def test_mdq_p2m_m2m_m2p_match_reference(oracle, ref_oracle):
    rng = np.random.default_rng(21)
    n = 160
    x, y, z = (rng.uniform(0, 1, n) for _ in range(3))
    m = rng.uniform(-0.5, 0.5, n)
    c_o, q_o = oracle.mdq_p2m(x, y, z, m)
    c_r, q_r = ref_oracle.mdq_p2m(x, y, z, m)
    assert np.allclose(c_o, c_r, rtol=1e-13, atol=1e-15) and np.allclose(q_o, q_r, rtol=1e-12, atol=1e-14)
    assert abs(q_r[8]) + abs(q_r[9]) + abs(q_r[10]) > 1e-3  # signed masses: a real dipole
    # M2M of eight sub-expansions equals the direct expansion (cartesian_qpole.cpp:180-239)
    cs, qs = [], []
    for k in range(8):
        sl = slice(20 * k, 20 * (k + 1))
        c, q = ref_oracle.mdq_p2m(x[sl], y[sl], z[sl], m[sl])
        cs.append(c)
        qs.append(q)
    comp_r = ref_oracle.mdq_m2m(np.array(cs), np.array(qs), c_r)
    comp_o = oracle.mdq_m2m(np.array(cs), np.array(qs), c_r)
    assert np.allclose(comp_o, comp_r, rtol=1e-12, atol=1e-14)
    assert np.allclose(comp_r, q_r, rtol=1e-9, atol=1e-10)
    for t in ([-8.0, 0.0, 0.0], [3.0, 2.5, -4.0]):
        a_o = oracle.mdq_m2p(t, c_r, q_r)
        a_r = ref_oracle.mdq_m2p(t, c_r, q_r)
        assert np.allclose(a_o, a_r, rtol=1e-13, atol=1e-16)
        # and approximates the direct sum (cartesian_qpole.cpp:130-172)
        d = np.array([x - t[0], y - t[1], z - t[2]])
        r = np.sqrt((d * d).sum(0))
        direct = np.array([-(m / r).sum(), *(m * d / r ** 3).sum(1)])
        assert np.allclose(a_r, direct, atol=1e-3)


def test_fixtures_regenerate_from_the_reference(ref_oracle):
    """every committed golden case is what the reference's own CPU code (oracle/_ref) produces for the case's seeded
    inputs today: the fixtures are the reference's outputs, not the restatement's. Arrays are compared bit for bit;
    the total energies to 1e-5, since the reference sums them in an OpenMP reduction whose order follows the thread
    count"""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(os.path.dirname(__file__), "golden",
                                                                              "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    for kind, n, seed, bucket in mg.CASES:
        fresh = mg.make_case(ref_oracle, kind, n, seed, bucket)
        stored = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"case_{kind}_{n}.npz")))
        assert set(fresh) == set(stored), (kind, set(fresh) ^ set(stored))
        for k, v in fresh.items():
            if k.endswith("_u"):
                assert abs(float(v) - float(stored[k])) <= 1e-5 * abs(float(stored[k])), (kind, k)
            else:
                assert np.array_equal(np.asarray(v), stored[k]), (kind, k)


def _edge_sets():
    rng = np.random.default_rng(123)
    yield "empty", np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32), [0, 1, 0, 1, 0, 1], 16
    one = np.array([0.3], np.float32)
    yield "one", one, one, one, [0, 1, 0, 1, 0, 1], 16
    same = np.full(700, 0.25, np.float32)  # 700 coincident bodies: a deepest-level leaf above the bucket size
    yield "coincident", same, same, same, [0, 1, 0, 1, 0, 1], 64
    x, y, z = (rng.uniform(0, 1, 500).astype(np.float32) for _ in range(3))
    yield "bucket1", x, y, z, [0, 1, 0, 1, 0, 1], 1
    x = rng.uniform(0, 16, 2000).astype(np.float32)
    y, z = (rng.uniform(0, 0.01, 2000).astype(np.float32) for _ in range(2))
    yield "reduced_axes", x, y, z, [0, 16, 0, 0.01, 0, 0.01], 8


@pytest.mark.parametrize("name", ["empty", "one", "coincident", "bucket1", "reduced_axes"])
def test_reference_wrapper_agrees_on_edge_cases(oracle, ref_oracle, name):
    """the restatement equals the reference's own code on the edge cases its tests cover: no bodies, one body,
    coincident bodies, bucket size 1 and a box with reduced axes (keys, leaves, counts and the linked octree)"""
    x, y, z, box, bucket = next((s[1:] for s in _edge_sets() if s[0] == name))
    box = np.asarray(box, np.float32)
    k1, k2 = oracle.sfc_keys(x, y, z, box), ref_oracle.sfc_keys(x, y, z, box)
    assert np.array_equal(k1, k2)
    assert np.array_equal(oracle.box_dim_bits(box), ref_oracle.box_dim_bits(box))
    s1, o1 = oracle.sort_keys(k1)
    s2, o2 = ref_oracle.sort_keys(k2)
    assert np.array_equal(s1, s2) and np.array_equal(o1, o2)
    l1, c1 = oracle.octree_leaves(s1, bucket)
    l2, c2 = ref_oracle.octree_leaves(s1, bucket)
    assert np.array_equal(l1, l2) and np.array_equal(c1, c2)
    t1, t2 = oracle.octree_link(l1), ref_oracle.octree_link(l1)
    for k in t1:
        assert np.array_equal(np.asarray(t1[k]), np.asarray(t2[k])), k


@pytest.mark.parametrize("name", ["one", "coincident", "bucket1", "reduced_axes"])
def test_reference_wrapper_agrees_on_edge_case_upsweep_and_walk(oracle, ref_oracle, name):
    """centres, multipoles and MAC radii (float upsweep) and the CPU tree walk of the edge cases, against the
    reference's own code. The walk is compared on the complete groups of 16 targets: for a last partial group the
    reference's target box includes slots it never writes (ryoanji/src/ryoanji/nbody/traversal_cpu.hpp:180-190), so
    its result there depends on stale memory"""
    x, y, z, box, bucket = next((s[1:] for s in _edge_sets() if s[0] == name))
    box = np.asarray(box, np.float32)
    n = len(x)
    m = np.random.default_rng(5).uniform(0.5, 1.5, n).astype(np.float32) / n
    h = np.full(n, 0.01, np.float32)
    s, order = oracle.sort_keys(oracle.sfc_keys(x, y, z, box))
    leaves, counts = oracle.octree_leaves(s, bucket)
    tree = oracle.octree_link(leaves)
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    xs, ys, zs, ms, hs = (a[order] for a in (x, y, z, m, h))
    c1, q1 = oracle.upsweep(xs, ys, zs, ms, layout, tree, 0.5, box)
    c2, q2 = ref_oracle.upsweep(xs, ys, zs, ms, layout, tree, 0.5, box)
    assert np.array_equal(c1, c2) and np.array_equal(q1, q2)
    g1 = oracle.gravity_cpu(tree, c1, q1, layout, xs, ys, zs, hs, ms, box)
    g2 = ref_oracle.gravity_cpu(tree, c2, q2, layout, xs, ys, zs, hs, ms, box)
    full = n - n % 16
    for a, b in zip(g1[1:], g2[1:]):
        assert np.array_equal(a[:full], b[:full])
    if full == n:
        assert abs(g1[0] - g2[0]) <= 1e-5 * max(abs(g2[0]), 1e-30)


@pytest.mark.parametrize("shells,lcut,hcut", [(0, 2.6, 2.8), (1, 2.6, 2.8), (2, 3.2, 3.0), (1, 1.5, 1.6)])
def test_ewald_restatement_against_reference_settings(oracle, ref_oracle, shells, lcut, hcut):
    """the root-multipole Ewald correction against the reference's own code at other replica shells and cut-offs,
    in an offset box of length 3 (ryoanji/src/ryoanji/nbody/ewald.hpp:200-389); hCut stays within the reference's
    ceil(hCut) <= 3"""
    rng = np.random.default_rng(17 + shells)
    n = 300
    x, y, z = (rng.uniform(-1.0, 2.0, n) for _ in range(3))
    m = rng.uniform(0.5, 1.5, n) / n
    box = np.array([-1.0, 2.0, -1.0, 2.0, -1.0, 2.0])
    c, q = oracle.p2m(x, y, z, m)
    rc, mr = np.asarray(c[:3], np.float64), np.asarray(q, np.float64)
    u1, *f1 = oracle.ewald(rc, mr, x, y, z, m, box, G=1.0, replica_shells=shells, lcut=lcut, hcut=hcut)
    u2, *f2 = ref_oracle.ewald(rc, mr, x, y, z, m, box, G=1.0, replica_shells=shells, lcut=lcut, hcut=hcut)
    for a, b in zip(f1, f2):
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())
    assert abs(u1 - u2) <= 1e-12 * abs(u2)
