"""Separate targets (ryo_solve_targets_f32): the field of a solve's tree at other points.

- The solve's own sorted bodies as targets give back its results bit for bit (same order, same fixed groups),
  open and periodic.
- A shuffled subset of bodies and arbitrary points off the bodies agree with FP64 direct sums at BH accuracy.
"""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _solve(p, params):
    import ryoanji_b200 as ryo
    ctx = ryo.Context(0)
    arrs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    n = p.n
    out = [torch.empty(n, device="cuda") for _ in range(4)]
    r = ryo.solve(*arrs, *out, params=params, ctx=ctx)
    return ctx, arrs, out, r


@pytest.mark.parametrize("kind", ["open", "periodic"])
def test_own_bodies_as_targets_reproduce_the_solve(kind):
    import ryoanji_b200 as ryo
    if kind == "open":
        p = ds.plummer(30000, seed=5, velocities=False)
        params = ryo.SolveParams(theta=0.5)
    else:
        p = ds.periodic_box(20000, seed=6, eps=0.002)
        params = ryo.SolveParams(theta=0.5, box=ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3))
    ctx, (x, y, z, m, h), out, r = _solve(p, params)
    (tp, tax, tay, taz), st = ryo.solve_targets(x, y, z, m, h, ctx=ctx)
    for got, want in zip((tp, tax, tay, taz), out):
        assert torch.equal(got, want)
    assert st.sum_p2p == r.sum_p2p and st.sum_m2p == r.sum_m2p
    assert st.potential_energy == pytest.approx(r.potential_energy, rel=1e-9)


def test_shuffled_subset_and_free_points_against_direct_sums():
    import ryoanji_b200 as ryo
    p = ds.plummer(40000, seed=7, velocities=False)
    ctx, (x, y, z, m, h), out, r = _solve(p, ryo.SolveParams(theta=0.5))
    n = p.n
    rng = np.random.default_rng(3)
    idx = torch.from_numpy(rng.choice(n, 3000, replace=False)).cuda()
    (tp, tax, tay, taz), _ = ryo.solve_targets(x[idx], y[idx], z[idx], m[idx], h[idx], ctx=ctx)
    rp, rx, ry, rz = ryo.direct_targets_f64(idx, x, y, z, m, h)
    a = torch.stack([tax, tay, taz], 1).double()
    ref = torch.stack([rx, ry, rz], 1)
    err = (torch.linalg.norm(a - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy()
    assert np.percentile(err, 99) < 2e-3 and np.median(err) < 2e-4, (np.percentile(err, 99), np.median(err))
    perr = (tp.double() - rp).abs() / rp.abs()
    assert float(perr.max()) < 1e-3

    # points that are not bodies, no masses or softening given: compare with a direct sum in which they are
    # appended as massless bodies
    k = 2000
    pts = [torch.from_numpy(rng.uniform(-1.5, 1.5, k).astype(np.float32)).cuda() for _ in range(3)]
    (_, fax, fay, faz), _ = ryo.solve_targets(*pts, ctx=ctx)
    X, Y, Z = (torch.cat([a, b]) for a, b in zip((x, y, z), pts))
    M = torch.cat([m, torch.zeros(k, device="cuda")])
    H = torch.cat([h, torch.full((k,), 1e-7, device="cuda")])  # a point meets itself at r = 0: keep 0 * 1/0 out
    tgt = torch.arange(n, n + k, device="cuda")
    _, rx, ry, rz = ryo.direct_targets_f64(tgt, X, Y, Z, M, H)
    a = torch.stack([fax, fay, faz], 1).double()
    ref = torch.stack([rx, ry, rz], 1)
    err = (torch.linalg.norm(a - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy()
    assert np.percentile(err, 99) < 2e-3, np.percentile(err, 99)


def test_targets_need_a_solve_first():
    import ryoanji_b200 as ryo
    ctx = ryo.Context(0)
    x = torch.zeros(8, device="cuda")
    with pytest.raises(ryo.RyoError):
        ryo.solve_targets(x, x, x, ctx=ctx)
