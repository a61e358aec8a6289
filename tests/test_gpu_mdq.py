"""Monopole + dipole + quadrupole expansions (CartesianMDQpole) in the solve.

- Signed masses, the reference's own test setting (ryoanji/test/nbody/traversal_cpu.cpp:27-140: Gaussian bodies,
  masses +-1/N, theta 0.2, bucket 64): 99th-percentile error < 3e-3, maximum < 3e-2 against the FP64 direct sum,
  potential energy within 1e-2; the quadrupole-only expansion is worse there.
- Every node's moments equal the exact FP64 expansion of its bodies (restated P2M, pinned to the reference).
- Positive masses: the dipole vanishes and the result equals the quadrupole solve to float rounding.
- The interaction lists do not depend on the expansion type.
"""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _signed_gaussian(n, seed):
    p = ds.gaussian(n, seed=seed, sigma=0.2)
    m = np.full(n, 1.0 / n)
    m[1::2] *= -1.0
    p.m = m.astype(np.float32)
    p.h = np.full(n, 0.002, np.float32)
    return p


def _run(p, multipole, theta):
    import ryoanji_b200 as ryo
    x, y, z, m, h = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (p.x, p.y, p.z, p.m, p.h))
    n = p.n
    pot, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    params = ryo.SolveParams(theta=theta, bucket_size=64, box=ryo.Box.cube(-1.0, 1.0), multipole=multipole)
    r = ryo.solve(x, y, z, m, h, pot, ax, ay, az, params)
    return r, (x, y, z, m, h), (pot, ax, ay, az)


def test_signed_masses_reference_bounds():
    import ryoanji_b200 as ryo
    p = _signed_gaussian(100000, 31)
    errs = {}
    for kind in ("quadrupole", "mdq"):
        r, (x, y, z, m, h), (pot, ax, ay, az) = _run(p, kind, 0.2)
        tgt = torch.arange(p.n, device="cuda")
        rp, rx, ry, rz = ryo.direct_targets_f64(tgt, x, y, z, m, h)
        a = torch.stack([ax, ay, az], 1).double()
        ref = torch.stack([rx, ry, rz], 1)
        d = (torch.linalg.norm(a - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy()
        errs[kind] = (float(np.percentile(d, 99)), float(d.max()))
        if kind == "mdq":
            e_ref = 0.5 * float(rp.sum())
            assert abs(r.potential_energy - e_ref) / abs(e_ref) < 1e-2
            assert errs[kind][0] < 3e-3 and errs[kind][1] < 3e-2, errs
    assert errs["mdq"][0] < errs["quadrupole"][0], errs


def test_node_moments_equal_exact_expansions(oracle):
    import ryoanji_b200 as ryo
    p = _signed_gaussian(30000, 32)
    r, (x, y, z, m, h), _ = _run(p, "mdq", 0.5)
    arr = ryo.solve_arrays()
    host = lambda t: np.ascontiguousarray(t.cpu().numpy())  # noqa: E731
    xs, ys, zs, ms = (host(t).astype(np.float64) for t in (x, y, z, m))
    links = host(arr["links"])
    cen, mp, dp = host(arr["centers"]), host(arr["multipoles"]), host(arr["dipoles"])
    child = host(arr["childOffsets"])
    nn = arr["numNodes"]

    def body_range(node):
        # first body of the first leaf below, one past the last body of the last leaf below
        lo = hi = node
        while child[lo] != 0:
            lo = child[lo]
        while child[hi] != 0:
            hi = child[hi] + 7
        return links[lo, 1], links[hi, 1] + links[hi, 2]

    rng = np.random.default_rng(1)
    nodes = [0] + list(rng.choice(nn, 400, replace=False))
    L = 2.0
    for node in nodes:
        b0, b1 = body_range(int(node))
        if b1 <= b0:
            continue
        c, q = oracle.mdq_p2m(xs[b0:b1], ys[b0:b1], zs[b0:b1], ms[b0:b1])
        w = np.abs(ms[b0:b1]).sum()
        assert np.allclose(cen[node, :3], c[:3], atol=1e-6 * L)
        got = np.concatenate([mp[node], dp[node, :3]])
        want = q[:11]
        scale = np.array([w] + [3 * w * L * L] * 7 + [w * L] * 3)
        assert np.all(np.abs(got - want) <= 2e-6 * scale + 1e-9), (node, got, want)


def test_positive_masses_and_interaction_lists():
    p = ds.plummer(50000, seed=33, velocities=False)
    rq, _, oq = _run(p, "quadrupole", 0.5)
    rm, _, om = _run(p, "mdq", 0.5)
    assert rq.sum_p2p == rm.sum_p2p and rq.sum_m2p == rm.sum_m2p
    a_q = torch.stack(oq[1:], 1)
    a_m = torch.stack(om[1:], 1)
    rel = (torch.linalg.norm(a_q - a_m, dim=1) / torch.linalg.norm(a_q, dim=1)).max()
    assert float(rel) < 2e-5, float(rel)


def test_step_flow_matches_reference_cpu_upsweep_and_direct_sums(ref_oracle_or_skip):
    """TreeBuilder + the individual steps with 12-float multipoles, then traverse(mdq=True): moments against the
    reference's own CPU upsweep of the same tree, forces against the FP64 direct sum"""
    import ryoanji_b200 as ryo
    ref = ref_oracle_or_skip
    p = _signed_gaussian(40000, 34)
    box = ryo.Box.cube(-1.0, 1.0)
    x, y, z, m, h = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (p.x, p.y, p.z, p.m, p.h))
    tb = ryo.TreeBuilder(64)
    nn = tb.update(x, y, z, box)
    order = tb.order().long()
    m, h = m[order].contiguous(), h[order].contiguous()
    centers = torch.zeros(nn, 4, device="cuda")
    mp = torch.zeros(nn, 12, device="cuda")
    ryo.compute_leaf_source_center(x, y, z, m, tb.leafToInternal(), tb.layout(), centers)
    ryo.upsweep_centers(tb.maxTreeLevel, tb.levelRange, tb.childOffsets(), centers)
    ryo.compute_leaf_multipoles(x, y, z, m, tb.leafToInternal(), tb.layout(), centers, mp, mdq=True)
    lr = tb.levelRange
    for level in range(tb.maxTreeLevel - 1, -1, -1):
        ryo.upsweep_multipoles(lr[level], lr[level + 1], tb.childOffsets(), centers, mp, mdq=True)
    ryo.set_mac(tb.nodeKeys(), centers, 1.0 / 0.2, box)

    host = lambda t: np.ascontiguousarray(t.cpu().numpy())  # noqa: E731
    nl = tb.numLeafNodes
    ni = (nl - 1) // 7
    tree = dict(numNodes=nn, numLeaves=nl, numInternal=ni, childOffsets=host(tb.childOffsets()),
                levelRange=np.asarray(tb.levelRange, np.int32), prefixes=host(tb.nodeKeys()).view(np.uint64),
                leafToInternal=np.concatenate([np.zeros(ni, np.int32), host(tb.leafToInternal())]))
    layout = host(tb.layout()).view(np.uint32)
    xs, ys, zs, ms = (host(t) for t in (x, y, z, m))
    c_ref, mp_ref = ref.upsweep_mdq(xs, ys, zs, ms, layout, tree, 0.2, [-1, 1, -1, 1, -1, 1])
    got = host(mp)
    w = np.abs(ms).sum()
    scale = np.array([w] + [3 * w * 4.0] * 7 + [w * 2.0] * 3 + [1.0])
    # the reference sums in float, the steps in double: compare at float-accumulation level
    assert np.all(np.abs(got - mp_ref) <= 1e-4 * scale + 1e-9), np.abs(got - mp_ref).max(0)

    groups = ryo.compute_fixed_groups(0, p.n, 64)
    pot, ax, ay, az = (torch.zeros(p.n, device="cuda") for _ in range(4))
    ryo.traverse(groups, 1, x, y, z, m, h, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(), tb.layout(),
                 centers, mp, 1.0, 0, (0.0, 0.0, 0.0), pot, ax, ay, az, mdq=True)
    tgt = torch.from_numpy(np.random.default_rng(4).choice(p.n, 4000, replace=False)).cuda()
    _, rx, ry, rz = ryo.direct_targets_f64(tgt, x, y, z, m, h)
    a = torch.stack([ax[tgt], ay[tgt], az[tgt]], 1).double()
    r = torch.stack([rx, ry, rz], 1)
    d = (torch.linalg.norm(a - r, dim=1) / torch.linalg.norm(r, dim=1)).cpu().numpy()
    assert np.percentile(d, 99) < 3e-3 and d.max() < 3e-2, (np.percentile(d, 99), d.max())


@pytest.fixture
def ref_oracle_or_skip():
    import sys
    import os
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if not pyoracle.have_reference():
        pytest.skip("reference wrapper not built")
    return pyoracle.Oracle(reference=True)
