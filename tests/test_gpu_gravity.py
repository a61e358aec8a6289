"""GPU parity of the gravity phases: upsweep, traversal, Ewald, direct sums, fused solve.

Tiers:
- bit for bit: per-group interaction counts (cells approximated, bodies summed directly) against the oracle's
  statement of the reference rule, evaluated on the same tree, centres and MAC radii; MAC radii against the oracle
  wherever the float centre is the same;
- tolerance: accelerations against the same interactions evaluated in double precision (relative 1e-5, float
  accumulation and rsqrt.approx), against the reference's CPU tree walk at the Barnes-Hut error level, and against
  the FP64 direct sum (1st-percentile relative error <= 1e-3 at theta = 0.5).
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


def host(t):
    return t.cpu().numpy()


def rel_err(ax, ay, az, rx, ry, rz):
    num = np.sqrt((ax - rx) ** 2 + (ay - ry) ** 2 + (az - rz) ** 2)
    den = np.sqrt(rx ** 2 + ry ** 2 + rz ** 2)
    return num / np.maximum(den, 1e-300)


@pytest.fixture(scope="module", params=CASES, ids=IDS)
def case(request):
    return dict(np.load(request.param))


def reference_flow(case, theta=0.5):
    """TreeBuilder + the reference's individual upsweep steps (ryoanji/test/demo.cu:319-346)"""
    import ryoanji_b200 as ryo
    box = ryo.Box(*[float(v) for v in case["box"]])
    o = case["order"]
    x, y, z = dev(case["x"]), dev(case["y"]), dev(case["z"])
    m, h = dev(case["m"][o]), dev(case["h"][o])
    tb = ryo.TreeBuilder(int(case["bucket"]))
    nn = tb.update(x, y, z, box)
    centers = torch.zeros(nn, 4, device="cuda")
    mp = torch.zeros(nn, 8, device="cuda")
    ryo.compute_leaf_source_center(x, y, z, m, tb.leafToInternal(), tb.layout(), centers)
    ryo.upsweep_centers(tb.maxTreeLevel, tb.levelRange, tb.childOffsets(), centers)
    ryo.compute_leaf_multipoles(x, y, z, m, tb.leafToInternal(), tb.layout(), centers, mp)
    lr = tb.levelRange
    for level in range(tb.maxTreeLevel - 1, -1, -1):
        ryo.upsweep_multipoles(lr[level], lr[level + 1], tb.childOffsets(), centers, mp)
    ryo.set_mac(tb.nodeKeys(), centers, 1.0 / theta, box)
    return tb, box, (x, y, z, m, h), centers, mp


def oracle_tree(case):
    ni = (len(case["counts"]) - 1) // 7
    return dict(childOffsets=case["tree_childOffsets"], internalToLeaf=case["tree_internalToLeaf"],
                parents=case["tree_parents"], numLeaves=len(case["counts"]), numInternal=ni,
                numNodes=len(case["tree_prefixes"]), prefixes=case["tree_prefixes"],
                levelRange=case["tree_levelRange"], leafToInternal=case["tree_leafToInternal"])


def test_upsweep_steps_match_double_oracle(oracle, case):
    tb, box, (x, y, z, m, h), centers, mp = reference_flow(case)
    t = oracle_tree(case)
    o = case["order"]
    c_ref, m_ref = oracle.upsweep(case["x"][o], case["y"][o], case["z"][o], case["m"][o], case["layout"], t, 0.5,
                                  case["box"], mode=1)
    c, q = host(centers), host(mp)
    scale = np.abs(c_ref[:, :3]).max()
    assert np.abs(c[:, :3] - c_ref[:, :3]).max() <= 4e-7 * scale
    same = np.all(c[:, :3] == c_ref[:, :3], axis=1)
    assert same.mean() > 0.9
    # the MAC radius is bit-exact wherever the float centre is
    assert np.array_equal(c[same, 3], c_ref[same, 3])
    # quadrupole entries to float round-off of the node's largest moment (per node), or of mass * (box size)^2
    L = float(max(case["box"][1::2] - case["box"][0::2]))
    scale = np.maximum(np.abs(q[:, 1:]).max(axis=1), np.abs(m_ref[:, 1:]).max(axis=1))
    tol = 2e-6 * scale + 1e-9 * np.abs(m_ref[:, 0]) * L * L
    assert np.all(np.abs(q[:, 1:] - m_ref[:, 1:]).max(axis=1) <= tol)
    assert np.allclose(q[:, 0], m_ref[:, 0], rtol=1e-6, atol=0)


def test_traverse_counts_exact_and_forces(oracle, case):
    """reference-signature traverse: per-group counts bit-exact, forces vs double evaluation of the same lists"""
    import ryoanji_b200 as ryo
    tb, box, (x, y, z, m, h), centers, mp = reference_flow(case)
    n = x.numel()
    groups = ryo.compute_fixed_groups(0, n, ryo.bh_max_target_size())
    periodic = case["box"][0] == 0 and case["box"][1] == 1 and len(case["x"]) == 1024
    shells = 1 if periodic else 0
    L = box.lengths
    p, ax, ay, az = (torch.zeros(n, device="cuda") for _ in range(4))
    pot, gm, gp = ryo.traverse(groups, 1, x, y, z, m, h, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(),
                               tb.layout(), centers, mp, 1.0, shells, L, p, ax, ay, az, group_counts=True)
    g = host(groups)
    hx, hy, hz, hm, hh = host(x), host(y), host(z), host(m), host(h)
    m2p, p2p, acc = oracle.traverse_rule(g[:-1], g[1:], hx, hy, hz, hh, hm,
                                         dict(childOffsets=host(tb.childOffsets()),
                                              internalToLeaf=host(tb.internalToLeaf())),
                                         host(tb.layout()).view(np.uint32), host(centers), host(mp), init_node=1,
                                         numShells=shells, boxL=L, evaluate=True)
    assert np.array_equal(host(gm).view(np.uint32), m2p)
    assert np.array_equal(host(gp).view(np.uint32), p2p)
    stats = ryo.read_bh_stats()
    sizes = np.diff(g)
    assert stats[0] == int((p2p.astype(np.int64) * sizes).sum()) and stats[1] == int(p2p.max())
    assert stats[2] == int((m2p.astype(np.int64) * sizes).sum()) and stats[3] == int(m2p.max())
    e = rel_err(host(ax), host(ay), host(az), acc[:, 1], acc[:, 2], acc[:, 3])
    assert np.percentile(e, 99) < 2e-6 and e.max() < 5e-5
    assert np.allclose(host(p), hm * acc[:, 0], rtol=1e-5, atol=1e-6 * np.abs(hm * acc[:, 0]).max())
    assert abs(pot - 0.5 * float((hm * acc[:, 0]).sum())) < 1e-5 * abs(pot)


def test_traverse_agrees_with_reference_cpu_walk(case):
    """the reference's CPU computeGravity on the same tree differs only by Barnes-Hut error (other groups)"""
    if "grav_ax" not in case:
        pytest.skip("no CPU walk")
    if case["h"].max() > 1e-3 and np.ptp(case["x"][case["order"]][:64]) < 1e-2:
        # softening (0.01) far above the clump size: the CPU walk's 16-body groups apply unsoftened multipoles
        # inside a clump where the 64-body groups sum softened bodies, so the two reference paths disagree
        pytest.skip("softening dominates the clumps")
    import ryoanji_b200 as ryo
    tb, box, (x, y, z, m, h), centers, mp = reference_flow(case)
    n = x.numel()
    groups = ryo.compute_fixed_groups(0, n, 64)
    p, ax, ay, az = (torch.zeros(n, device="cuda") for _ in range(4))
    ryo.traverse(groups, 1, x, y, z, m, h, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(), tb.layout(),
                 centers, mp, 1.0, 0, None, p, ax, ay, az)
    e = rel_err(host(ax), host(ay), host(az), case["grav_ax"], case["grav_ay"], case["grav_az"])
    assert np.percentile(e, 99) < 2e-3


def test_solve_matches_oracle_path(oracle):
    """fused solve: tree bit-exact, per-group counts bit-exact against the oracle rule on the solve's own nodes,
    forces against their double-precision evaluation"""
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    pset = ds.plummer(40000, seed=21, velocities=False)
    x, y, z, m, h = (dev(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h))
    n = x.numel()
    p, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx = ryo.Context()
    res = ryo.solve(x, y, z, m, h, p, ax, ay, az, ryo.SolveParams(theta=0.5), order=order, ctx=ctx)
    arr = ryo.solve_arrays(ctx)
    box = np.array(res.box, np.float32)
    keys = oracle.sfc_keys(pset.x, pset.y, pset.z, box)
    sk, o = oracle.sort_keys(keys)
    assert np.array_equal(host(order).view(np.uint32), o)
    assert np.array_equal(host(x), pset.x[o])
    l_ref, c_ref = oracle.octree_leaves(sk, 64)
    assert np.array_equal(host(arr["leaves"]).view(np.uint64), l_ref)
    t_ref = oracle.octree_link(l_ref)
    for k in ("prefixes", "childOffsets", "internalToLeaf", "parents"):
        assert np.array_equal(host(arr[k]).view(t_ref[k].dtype), t_ref[k]), k
    layout = np.concatenate([[0], np.cumsum(c_ref)]).astype(np.uint32)
    c_dbl, m_dbl = oracle.upsweep(pset.x[o], pset.y[o], pset.z[o], pset.m[o], layout, t_ref, 0.5, box, mode=1)
    cg, mg = host(arr["centers"]), host(arr["multipoles"])
    same = np.all(cg[:, :3] == c_dbl[:, :3], axis=1)
    assert same.mean() > 0.9 and np.array_equal(cg[same, 3], c_dbl[same, 3])
    assert np.abs(cg[:, :3] - c_dbl[:, :3]).max() <= 4e-7 * np.abs(c_dbl[:, :3]).max()
    g = host(arr["groups"])
    m2p, p2p, acc = oracle.traverse_rule(g[:-1], g[1:], host(x), host(y), host(z), host(h), host(m),
                                         dict(childOffsets=t_ref["childOffsets"],
                                              internalToLeaf=t_ref["internalToLeaf"]), layout, cg, mg, evaluate=True)
    assert np.array_equal(host(arr["groupM2P"]).view(np.uint32), m2p)
    assert np.array_equal(host(arr["groupP2P"]).view(np.uint32), p2p)
    e = rel_err(host(ax), host(ay), host(az), acc[:, 1], acc[:, 2], acc[:, 3])
    assert np.percentile(e, 99) < 2e-6 and e.max() < 5e-5
    assert res.sum_m2p == int((m2p.astype(np.int64) * np.diff(g)).sum())


def test_solve_upsweep_by_levels_matches_double_oracle(oracle):
    """a tree of more than 2^17 nodes (188k here), whose internal nodes the fused upsweep combines one level per
    launch instead of by the climb: links bit-exact, centres, MAC radii and multipoles against the FP64 oracle"""
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    pset = ds.plummer(400000, seed=22, velocities=False)
    x, y, z, m, h = (dev(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h))
    n = x.numel()
    p, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    ctx = ryo.Context()
    res = ryo.solve(x, y, z, m, h, p, ax, ay, az, ryo.SolveParams(theta=0.5, bucket_size=8), ctx=ctx)
    assert res.num_nodes > 1 << 17
    arr = ryo.solve_arrays(ctx)
    box = np.array(res.box, np.float32)
    sk, o = oracle.sort_keys(oracle.sfc_keys(pset.x, pset.y, pset.z, box))
    l_ref, c_ref = oracle.octree_leaves(sk, 8)
    t_ref = oracle.octree_link(l_ref)
    for k in ("prefixes", "childOffsets", "internalToLeaf", "parents"):
        assert np.array_equal(host(arr[k]).view(t_ref[k].dtype), t_ref[k]), k
    layout = np.concatenate([[0], np.cumsum(c_ref)]).astype(np.uint32)
    c_dbl, m_dbl = oracle.upsweep(pset.x[o], pset.y[o], pset.z[o], pset.m[o], layout, t_ref, 0.5, box, mode=1)
    cg, mg = host(arr["centers"]), host(arr["multipoles"])
    assert np.abs(cg[:, :3] - c_dbl[:, :3]).max() <= 4e-7 * np.abs(c_dbl[:, :3]).max()
    same = np.all(cg[:, :3] == c_dbl[:, :3], axis=1)
    assert same.mean() > 0.9 and np.array_equal(cg[same, 3], c_dbl[same, 3])
    L = float(max(box[1::2] - box[0::2]))
    scale = np.maximum(np.abs(mg[:, 1:]).max(axis=1), np.abs(m_dbl[:, 1:]).max(axis=1))
    tol = 2e-6 * scale + 1e-9 * np.abs(m_dbl[:, 0]) * L * L
    assert np.all(np.abs(mg[:, 1:] - m_dbl[:, 1:]).max(axis=1) <= tol)
    assert np.allclose(mg[:, 0], m_dbl[:, 0], rtol=1e-6, atol=0)


SPLIT_COST = 32768  # direct bodies + 2 x approximated cells past which the traversal splits a group over warps


def test_heavy_groups_split_over_warps(oracle):
    """groups whose interaction lists are too long for one warp (sparse outskirts of a Plummer sphere whose bounding
    box reaches the centre) are evaluated by several warps in a second pass: per-group counts stay bit-exact, forces
    match the double evaluation of the same lists, and a repeated solve gives identical results"""
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    pset = ds.plummer(100000, seed=1, velocities=False)
    ctx = ryo.Context()
    runs = []
    for _ in range(2):
        x, y, z, m, h = (dev(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h))
        n = x.numel()
        out = [torch.empty(n, device="cuda") for _ in range(4)]
        res = ryo.solve(x, y, z, m, h, *out, ryo.SolveParams(theta=0.5), ctx=ctx)
        runs.append(out)
    for a, b in zip(*runs):
        assert torch.equal(a, b)
    p, ax, ay, az = runs[-1]
    arr = ryo.solve_arrays(ctx)
    g = host(arr["groups"]).view(np.uint32)
    gm, gp = host(arr["groupM2P"]).view(np.uint32), host(arr["groupP2P"]).view(np.uint32)
    heavy = gp.astype(np.int64) + 2 * gm.astype(np.int64) > SPLIT_COST
    assert heavy.sum() >= 1 and res.max_p2p > SPLIT_COST // 2
    tree = dict(childOffsets=host(arr["childOffsets"]), internalToLeaf=host(arr["internalToLeaf"]))
    cg = np.ascontiguousarray(host(arr["centers"]))
    mg = np.ascontiguousarray(host(arr["multipoles"]))
    hx, hy, hz, hm, hh = host(x), host(y), host(z), host(m), host(h)
    m2p, p2p, acc = oracle.traverse_rule(g[:-1], g[1:], hx, hy, hz, hh, hm, tree, host(arr["layout"]).view(np.uint32),
                                         cg, mg, evaluate=True)
    assert np.array_equal(gm, m2p) and np.array_equal(gp, p2p)
    sizes = np.diff(g).astype(np.int64)
    assert res.sum_p2p == int((p2p.astype(np.int64) * sizes).sum()) and res.max_p2p == int(p2p.max())
    e = rel_err(host(ax), host(ay), host(az), acc[:, 1], acc[:, 2], acc[:, 3])
    assert np.percentile(e, 99) < 2e-6 and e.max() < 5e-5
    for k in np.flatnonzero(heavy):  # the split groups themselves
        assert e[g[k]:g[k + 1]].max() < 5e-6, k
    assert np.allclose(host(p), hm * acc[:, 0], rtol=1e-5, atol=1e-6 * np.abs(hm * acc[:, 0]).max())
    assert res.potential_energy == pytest.approx(0.5 * float((hm * acc[:, 0]).sum()), rel=1e-5)


@pytest.mark.parametrize("kind", ["plummer", "cube", "halos"])
def test_solve_accuracy_vs_fp64_direct(kind):
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    n = 1 << 15
    if kind == "plummer":
        pset = ds.plummer(n, seed=1, velocities=False)
    elif kind == "cube":
        pset = ds.uniform_cube(n, seed=2)
    else:
        pset = ds.hernquist_halos(n, num_halos=16, seed=3)
    x, y, z, m, h = (dev(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h))
    p, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    res = ryo.solve(x, y, z, m, h, p, ax, ay, az, ryo.SolveParams(theta=0.5))
    targets = torch.from_numpy(np.random.default_rng(0).choice(n, 2048, replace=False)).cuda()
    rp, rx, ry, rz = ryo.direct_targets_f64(targets, x, y, z, m, h)
    t = targets
    e = rel_err(host(ax[t]).astype(np.float64), host(ay[t]), host(az[t]), host(rx), host(ry), host(rz))
    assert np.percentile(e, 99) < 1e-3, np.percentile(e, 99)
    assert np.median(e) < 2e-4
    # potential energy from the tree against the direct potential of the sample
    assert np.allclose(host(p[t]), host(rp), rtol=5e-3, atol=1e-3 * np.abs(host(rp)).max())
    assert res.potential_energy < 0


def test_overflow_split_retry(oracle):
    """groups that overflow a (deliberately small) stack are split and traversed again with identical results
    (ryoanji/test/interface/traversal_overflow_gpu.cpp:39-116: a spread grid group and a compact group)"""
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    src = ds.gaussian(20000, seed=8, sigma=0.3)
    src.h[:] = 1e-6
    box = ryo.Box.cube(-1.0, 1.0)
    x, y, z, m, h = (dev(a) for a in (src.x, src.y, src.z, src.m, src.h))
    tb = ryo.TreeBuilder(16)
    nn = tb.update(x, y, z, box)
    perm = tb.order().long()
    m, h = m[perm].contiguous(), h[perm].contiguous()
    centers = torch.zeros(nn, 4, device="cuda")
    mp = torch.zeros(nn, 8, device="cuda")
    ryo.compute_leaf_source_center(x, y, z, m, tb.leafToInternal(), tb.layout(), centers)
    ryo.upsweep_centers(21, tb.levelRange, tb.childOffsets(), centers)
    ryo.compute_leaf_multipoles(x, y, z, m, tb.leafToInternal(), tb.layout(), centers, mp)
    lr = tb.levelRange
    for level in range(20, -1, -1):
        ryo.upsweep_multipoles(lr[level], lr[level + 1], tb.childOffsets(), centers, mp)
    ryo.set_mac(tb.nodeKeys(), centers, 2.0, box)
    nt = 128
    xt = np.zeros(nt, np.float32)
    yt = np.zeros(nt, np.float32)
    zt = np.zeros(nt, np.float32)
    for i in range(64):
        xt[i], yt[i], zt[i] = -0.9 + 0.6 * (i % 4), -0.9 + 0.6 * ((i // 4) % 4), -0.9 + 0.6 * (i // 16)
    for i in range(64, nt):
        xt[i], yt[i], zt[i] = 0.1 + 1e-3 * (i - 64) / 63, 0.1, 0.1
    XT, YT, ZT = dev(xt), dev(yt), dev(zt)
    MT, HT = torch.zeros(nt, device="cuda"), torch.full((nt,), 1e-6, device="cuda")
    groups = torch.tensor([0, 64, nt], dtype=torch.int32, device="cuda")

    def run(cap):
        a = [torch.zeros(nt, device="cuda") for _ in range(3)]
        ryo.traverse(groups, 1, XT, YT, ZT, MT, HT, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(),
                     tb.layout(), centers, mp, 1.0, 0, None, None, *a, stack_capacity=cap)
        return [host(v) for v in a], ryo.read_traversal_retries()

    base, r0 = run(0)
    assert r0 == 0
    found = False
    for cap in (48, 64, 96, 128, 192, 256):
        try:
            acc, retries = run(cap)
        except ryo.RyoError as e:
            assert e.status == 4  # a single target overflowed: try a larger stack
            continue
        if retries > 0:
            found = True
            # split groups see other bounding boxes and so apply a different (equally valid) approximation:
            # they are checked against the direct sum below, like the reference test
            base = acc
            break
    assert found, "no stack capacity produced a split-and-retry"
    # and against the direct sum (the reference test's 1e-2 bound)
    hx, hy, hz, hm, hh = host(x), host(y), host(z), host(m), host(h)
    d = oracle.direct  # double-precision direct sum of the sources on the probes (probes carry no mass)
    xs_all = np.concatenate([hx, xt]).astype(np.float32)
    ys_all = np.concatenate([hy, yt]).astype(np.float32)
    zs_all = np.concatenate([hz, zt]).astype(np.float32)
    hs_all = np.concatenate([hh, np.full(nt, 1e-6, np.float32)]).astype(np.float32)
    ms_all = np.concatenate([hm, np.zeros(nt, np.float32)]).astype(np.float32)
    pot, rx, ry, rz = d(xs_all, ys_all, zs_all, hs_all, ms_all, np.arange(len(hx), len(hx) + nt))
    e = rel_err(*base, rx, ry, rz)
    assert e.max() < 1e-2


def test_ewald_matches_oracle(oracle, case):
    if "ewald_ax" not in case:
        pytest.skip("not periodic")
    import ryoanji_b200 as ryo
    o = case["order"]
    x, y, z, m = (dev(case[k][o]) for k in ("x", "y", "z", "m"))
    n = x.numel()
    groups = ryo.compute_fixed_groups(0, n, 64)
    p, ax, ay, az = (torch.zeros(n, device="cuda") for _ in range(4))
    box = ryo.Box.cube(0.0, 1.0, ryo.BOUNDARY_PERIODIC)
    u = ryo.compute_gravity_ewald(case["centers"][0, :3], case["multipoles"][0], groups, x, y, z, m, box, 1.0, p, ax,
                                  ay, az)
    scale = np.abs(np.stack([case["ewald_ax"], case["ewald_ay"], case["ewald_az"]])).max()
    for a, k in ((ax, "ewald_ax"), (ay, "ewald_ay"), (az, "ewald_az")):
        assert np.abs(host(a) - case[k]).max() < 2e-5 * scale, k
    assert np.abs(host(p) - case["ewald_pot"]).max() < 2e-5 * np.abs(case["ewald_pot"]).max()
    assert abs(u - float(case["ewald_u"])) < 1e-5 * abs(float(case["ewald_u"]))


def test_ewald_requires_cubic_box():
    import ryoanji_b200 as ryo
    x = torch.zeros(64, device="cuda")
    g = ryo.compute_fixed_groups(0, 64, 64)
    with pytest.raises(ryo.RyoError) as e:
        ryo.compute_gravity_ewald([0, 0, 0], [1, 0, 0, 0, 0, 0, 0, 0], g, x, x, x, x,
                                  ryo.Box(0, 1, 0, 2, 0, 1, (1, 1, 1)), 1.0, None, x.clone(), x.clone(), x.clone())
    assert e.value.status == 7


def test_direct_sums(oracle, case):
    if "direct_ax" not in case:
        pytest.skip("no direct reference")
    import ryoanji_b200 as ryo
    o = case["order"]
    x, y, z, m, h = (case[k][o] for k in ("x", "y", "z", "m", "h"))
    n = len(x)
    X, Y, Z, M, H = (dev(a.astype(np.float64)) for a in (x, y, z, m, h))
    p, ax, ay, az = (torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4))
    ryo.direct_sum(0, n, n, [0.0, 0.0, 0.0], 0, X, Y, Z, M, H, p, ax, ay, az)
    for a, k in ((ax, "direct_ax"), (ay, "direct_ay"), (az, "direct_az"), (p, "direct_pot")):
        assert np.allclose(host(a), case[k], rtol=1e-10, atol=1e-10 * np.abs(case[k]).max()), k
    Xf, Yf, Zf, Mf, Hf = (dev(a) for a in (x, y, z, m, h))
    pf, axf, ayf, azf = (torch.zeros(n, device="cuda") for _ in range(4))
    ryo.direct_sum(0, n, n, [0.0, 0.0, 0.0], 0, Xf, Yf, Zf, Mf, Hf, pf, axf, ayf, azf)
    e = rel_err(host(axf), host(ayf), host(azf), case["direct_ax"], case["direct_ay"], case["direct_az"])
    assert e.max() < 1e-5
    t = torch.arange(0, n, 5, device="cuda")
    rp, rx, ry, rz = ryo.direct_targets_f64(t, Xf, Yf, Zf, Mf, Hf)
    idx = host(t)
    assert np.allclose(host(rx), case["direct_ax"][idx], rtol=1e-12, atol=1e-12 * np.abs(case["direct_ax"]).max())
    assert np.allclose(host(rp), case["direct_pot"][idx], rtol=1e-12, atol=1e-12 * np.abs(case["direct_pot"]).max())


def test_single_leaf_tree_solve():
    """N <= bucket: the root is the only node (the reference would read past the node arrays here)"""
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    pset = ds.plummer(50, seed=4, velocities=False)
    x, y, z, m, h = (dev(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h))
    p, ax, ay, az = (torch.empty(50, device="cuda") for _ in range(4))
    res = ryo.solve(x, y, z, m, h, p, ax, ay, az)
    assert res.num_nodes == 1 and res.sum_m2p == 0 and res.sum_p2p == 50 * 50
    t = torch.arange(50, device="cuda")
    rp, rx, ry, rz = ryo.direct_targets_f64(t, x, y, z, m, h)
    e = rel_err(host(ax), host(ay), host(az), host(rx), host(ry), host(rz))
    assert e.max() < 1e-5


def test_coincident_bodies_and_tiny_sets(oracle):
    """300 bodies at one point beside 5,000 others: their keys are equal, so one leaf at the deepest level holds more
    than the bucket size. Tree, per-group counts and forces against the oracle; then one and two bodies."""
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(4)
    pos = rng.uniform(-1, 1, (5300, 3)).astype(np.float32)
    pos[5000:] = np.float32(0.123456)
    hx, hy, hz = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    n = len(hx)
    hm = np.full(n, 1.0 / n, np.float32)
    hh = np.full(n, 0.01, np.float32)
    box6 = np.array([-1, 1] * 3, np.float32)
    x, y, z, m, h = (dev(a) for a in (hx, hy, hz, hm, hh))
    p, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx = ryo.Context()
    res = ryo.solve(x, y, z, m, h, p, ax, ay, az, ryo.SolveParams(theta=0.5, box=ryo.Box.cube(-1.0, 1.0)),
                    order=order, ctx=ctx)
    keys = oracle.sfc_keys(hx, hy, hz, box6)
    sk, o = oracle.sort_keys(keys)
    assert np.array_equal(host(order).view(np.uint32), o)
    l_ref, c_ref = oracle.octree_leaves(sk, 64)
    assert c_ref.max() == 300  # the coincident bodies share one leaf
    arr = ryo.solve_arrays(ctx)
    assert np.array_equal(host(arr["leaves"]).view(np.uint64), l_ref)
    g = host(arr["groups"]).view(np.uint32)
    tree = dict(childOffsets=host(arr["childOffsets"]), internalToLeaf=host(arr["internalToLeaf"]))
    m2p, p2p, acc = oracle.traverse_rule(g[:-1], g[1:], host(x), host(y), host(z), host(h), host(m), tree,
                                         host(arr["layout"]).view(np.uint32), np.ascontiguousarray(host(arr["centers"])),
                                         np.ascontiguousarray(host(arr["multipoles"])), evaluate=True)
    assert np.array_equal(host(arr["groupM2P"]).view(np.uint32), m2p)
    assert np.array_equal(host(arr["groupP2P"]).view(np.uint32), p2p)
    assert res.sum_p2p == int((p2p.astype(np.int64) * np.diff(g)).sum())
    gx, gy, gz = host(ax), host(ay), host(az)
    assert np.isfinite(gx).all() and np.isfinite(host(p)).all()
    # the coincident bodies pull each other with zero force; their acceleration is the rest's
    e = rel_err(gx, gy, gz, acc[:, 1], acc[:, 2], acc[:, 3])
    assert np.percentile(e, 99) < 2e-6 and e.max() < 5e-5

    for k in (1, 2):
        xs, ys, zs, ms, hs = (dev(a) for a in (hx[:k], hy[:k], hz[:k], hm[:k], hh[:k]))
        out = [torch.empty(k, device="cuda") for _ in range(4)]
        r = ryo.solve(xs, ys, zs, ms, hs, *out)
        assert r.sum_p2p == k * k and r.sum_m2p == 0
        t = torch.arange(k, device="cuda")
        rp, rx, ry, rz = ryo.direct_targets_f64(t, xs, ys, zs, ms, hs)
        for got, want in zip(out[1:], (rx, ry, rz)):
            assert np.allclose(host(got), host(want), rtol=1e-5, atol=1e-7)
        if k == 1:
            assert float(out[1].abs().max()) == 0.0
