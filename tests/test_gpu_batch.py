"""Batched solve: many systems in one launch per phase must give each system the result of its own solve.

The single-system solve is the reference-path composition (tested bit for bit against the oracle elsewhere); a
system inside a batch has the same box, tree (its leaves stop well above level 21 - L), groups and traversal order,
so its sorted bodies must be identical and its forces, potentials and energy equal to float rounding. (A group's
sums are bitwise those of its solve unless one of the two solves split the group over several warps and the other
did not: the split threshold follows the solve's size.)
"""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _systems(seed=0):
    out = []
    out.append(("plummer", ds.plummer(20000, seed=seed + 1, velocities=True), None))
    out.append(("cube", ds.uniform_cube(9000, seed=seed + 2, eps=0.002), None))
    p = ds.plummer(3000, seed=seed + 3, a=0.5, eps=0.005, velocities=True, center=(3.0, -1.0, 2.0))
    out.append(("offset", p, None))
    out.append(("periodic", ds.periodic_box(6000, seed=seed + 4, eps=0.001), "periodic"))
    g = ds.gaussian(1500, seed=seed + 5, sigma=0.1)
    out.append(("given-open", g, "open"))
    out.append(("tiny", ds.uniform_cube(40, seed=seed + 6, eps=0.01), None))
    out.append(("single", ds.uniform_cube(1, seed=seed + 7, eps=0.01), None))
    # sparse outskirts: some groups are split over several warps in a second traversal pass
    out.append(("outskirts", ds.plummer(100000, seed=1, velocities=True), None))
    return out


def _box_for(kind, p):
    import ryoanji_b200 as ryo
    if kind == "periodic":
        return ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    if kind == "open":
        lo = float(min(p.x.min(), p.y.min(), p.z.min())) - 0.01
        hi = float(max(p.x.max(), p.y.max(), p.z.max())) + 0.01
        return ryo.Box.cube(lo, hi)
    return None


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _vel(p):
    if p.vx is None:
        z = np.zeros(p.n, np.float32)
        return z, z.copy(), z.copy()
    return p.vx, p.vy, p.vz


def _run_batch(systems, params):
    import ryoanji_b200 as ryo
    cat = lambda f: _dev(np.concatenate([f(p) for _, p, _ in systems]))  # noqa: E731
    x, y, z = cat(lambda p: p.x), cat(lambda p: p.y), cat(lambda p: p.z)
    m, h = cat(lambda p: p.m), cat(lambda p: p.h)
    vx, vy, vz = (cat(lambda p, k=k: _vel(p)[k]) for k in range(3))
    n = x.numel()
    pot, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    desc = [ryo.BatchSystem(p.n, _box_for(kind, p)) for _, p, kind in systems]
    res = ryo.solve_batch(desc, x, y, z, m, h, pot, ax, ay, az, params, v=(vx, vy, vz), order=order)
    return res, dict(x=x, y=y, z=z, m=m, h=h, vx=vx, p=pot, ax=ax, ay=ay, az=az, order=order)


@pytest.mark.parametrize("tol", [0.0, 2.0], ids=["fixed-groups", "spatial-groups"])
def test_batch_equals_single_solves(tol):
    """with spatial groups each system's fixed windows are split with its own box, exactly as its single solve does"""
    import ryoanji_b200 as ryo
    systems = _systems()
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32, group_tolerance=tol)
    res, B = _run_batch(systems, params)
    assert res.stats.retries == 0
    first = 0
    groups = 0
    for (name, p, kind), e_batch, box in zip(systems, res.energies, res.boxes):
        n = p.n
        sl = slice(first, first + n)
        first += n
        x, y, z, m, h = (_dev(a) for a in (p.x, p.y, p.z, p.m, p.h))
        vx, vy, vz = (_dev(a) for a in _vel(p))
        pot, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
        order = torch.empty(n, dtype=torch.int32, device="cuda")
        given = _box_for(kind, p)
        sp = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32, box=given, num_shells=1, group_tolerance=tol)
        r = ryo.solve(x, y, z, m, h, pot, ax, ay, az, sp, v=(vx, vy, vz), order=order)
        groups += r.num_groups
        if given is None:
            assert r.box == pytest.approx(box, rel=0, abs=0), name  # the same enclosing cube, bit for bit
        assert torch.equal(B["order"][sl] - (first - n), order), name
        assert torch.equal(B["x"][sl], x) and torch.equal(B["z"][sl], z) and torch.equal(B["vx"][sl], vx), name
        # a group may be split over several warps in one solve and not in the other (the threshold follows the
        # solve's size), which moves its sums by a few float ulps: compare on the system's own field scale. A periodic
        # body's potential is a small remainder of large replica and Ewald terms, a few ulps of which are about 1e-5
        # of the remainder.
        amax = float(torch.sqrt(ax * ax + ay * ay + az * az).max()) + 1e-30
        for k, ref in (("ax", ax), ("ay", ay), ("az", az)):
            d = (B[k][sl] - ref).abs() / amax
            assert float(d.max()) <= 1e-6, (name, k, float(d.max()))
        dp = (B["p"][sl] - pot).abs() / (float(pot.abs().max()) + 1e-30)
        assert float(dp.max()) <= (1e-4 if kind == "periodic" else 1e-6), (name, float(dp.max()))
        assert e_batch == pytest.approx(r.potential_energy, rel=1e-4 if kind == "periodic" else 1e-7, abs=1e-12), name
    assert res.stats.num_groups == groups


def test_batch_mdq_signed_masses_equals_single_solves():
    """monopole + dipole + quadrupole expansions of signed masses (node dipoles, and an FP64 dipole in every system
    root): each system of the batch gets its single solve's result"""
    import ryoanji_b200 as ryo
    systems = []
    for i, (n, sigma) in enumerate(((20000, 0.2), (5000, 0.1), (700, 0.3))):
        p = ds.gaussian(n, seed=40 + i, sigma=sigma)
        m = np.full(n, 1.0 / n)
        m[1::2] *= -1.0
        p.m = m.astype(np.float32)
        p.h = np.full(n, 0.002, np.float32)
        systems.append((f"signed{i}", p, None))
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32, multipole="mdq")
    res, B = _run_batch(systems, params)
    first = 0
    for (name, p, _), e_batch, box in zip(systems, res.energies, res.boxes):
        n = p.n
        sl = slice(first, first + n)
        first += n
        x, y, z, m, h = (_dev(a) for a in (p.x, p.y, p.z, p.m, p.h))
        pot, ax, ay, az = (torch.empty(n, device="cuda") for _ in range(4))
        order = torch.empty(n, dtype=torch.int32, device="cuda")
        r = ryo.solve(x, y, z, m, h, pot, ax, ay, az, params, order=order)
        assert r.box == pytest.approx(box, rel=0, abs=0), name
        assert torch.equal(B["order"][sl] - (first - n), order), name
        assert torch.equal(B["x"][sl], x) and torch.equal(B["m"][sl], m), name
        # groups split over warps in one solve and not in the other move sums by a few ulps of their value
        amax = float(torch.sqrt(ax * ax + ay * ay + az * az).max()) + 1e-30
        for k, ref in (("ax", ax), ("ay", ay), ("az", az)):
            d = (B[k][sl] - ref).abs() / amax
            assert float(d.max()) <= 1e-6, (name, k, float(d.max()))
        dp = (B["p"][sl] - pot).abs() / (float(pot.abs().max()) + 1e-30)
        assert float(dp.max()) <= 1e-6, (name, float(dp.max()))
        assert e_batch == pytest.approx(r.potential_energy, rel=1e-6, abs=1e-9), name


def test_batch_many_small_systems_against_direct_sums():
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(11)
    sizes = [int(v) for v in rng.integers(1, 900, 300)]
    sizes[:4] = [1, 2, 63, 65]
    systems = [(f"s{i}", ds.plummer(s, seed=100 + i, velocities=False, center=tuple(rng.uniform(-5, 5, 3))), None)
               for i, s in enumerate(sizes)]
    params = ryo.SolveParams(theta=0.5, bucket_size=16, group_size=64)
    res, B = _run_batch(systems, params)
    assert len(res.energies) == 300
    first = 0
    worst = 0.0
    for (name, p, _), s in zip(systems, sizes):
        sl = slice(first, first + s)
        first += s
        if s < 2:
            assert float(B["ax"][sl].abs().max()) == 0.0
            continue
        x, y, z, m, h = (B[k][sl].contiguous() for k in ("x", "y", "z", "m", "h"))
        pd, axd, ayd, azd = (torch.zeros(s, device="cuda") for _ in range(4))
        ryo.direct_sum(0, s, s, (0.0, 0.0, 0.0), 0, x, y, z, m, h, pd, axd, ayd, azd)
        a = torch.sqrt(axd ** 2 + ayd ** 2 + azd ** 2)
        err = torch.sqrt((B["ax"][sl] - axd) ** 2 + (B["ay"][sl] - ayd) ** 2 + (B["az"][sl] - azd) ** 2) / a
        worst = max(worst, float(torch.quantile(err, 0.99)) if s > 100 else float(err.max()))
    assert worst < 5e-3, worst


def test_batch_rejects_bad_descriptions():
    import ryoanji_b200 as ryo
    x = torch.zeros(10, device="cuda")
    with pytest.raises(ryo.RyoError):
        ryo.solve_batch([ryo.BatchSystem(4), ryo.BatchSystem(4)], x, x, x, x, x, x, x, x, x)  # 8 != 10 bodies
    with pytest.raises(ryo.RyoError):
        ryo.solve_batch([ryo.BatchSystem(10), ryo.BatchSystem(0)], x, x, x, x, x, x, x, x, x)  # empty system
    with pytest.raises(ryo.RyoError):
        ryo.solve_batch([ryo.BatchSystem(1)] * 10 + [ryo.BatchSystem(0)], x, x, x, x, x, x, x, x, x)
    bad = ryo.Box(0, 1, 0, 2, 0, 1, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    with pytest.raises(ryo.RyoError):
        ryo.solve_batch([ryo.BatchSystem(10, bad)], x, x, x, x, x, x, x, x, x)


def test_batch_system_counts_between_powers_of_eight():
    """a batch of ns systems builds one tree whose system level holds 8^L >= ns nodes; the nodes past the last system
    are empty and own no per-system entry (box, root expansion). Batches of 9 and 65 systems (55 and 447 empty
    system-level nodes), solved one after the other so that each batch's per-system tables follow the previous one's
    in memory, each equal their systems' single solves"""
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(23)
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=64, group_tolerance=2.0)
    for ns in (65, 9, 65):
        sizes = [int(v) for v in rng.integers(200, 3000, ns)]
        systems = [(f"s{i}", ds.plummer(s, seed=300 + i, velocities=False, center=tuple(rng.uniform(-5, 5, 3))),
                    None) for i, s in enumerate(sizes)]
        res, B = _run_batch(systems, params)
        assert len(res.energies) == ns
        first = 0
        for (name, p, _), e_batch in zip(systems, res.energies):
            sl = slice(first, first + p.n)
            first += p.n
            x, y, z, m, h = (_dev(a) for a in (p.x, p.y, p.z, p.m, p.h))
            pot, ax, ay, az = (torch.empty(p.n, device="cuda") for _ in range(4))
            sp = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=64, group_tolerance=2.0)
            r = ryo.solve(x, y, z, m, h, pot, ax, ay, az, sp)
            assert torch.equal(B["x"][sl], x), (ns, name)
            amax = float(torch.sqrt(ax * ax + ay * ay + az * az).max()) + 1e-30
            for k, ref in (("ax", ax), ("ay", ay), ("az", az)):
                assert float(((B[k][sl] - ref).abs() / amax).max()) <= 1e-6, (ns, name, k)
            assert e_batch == pytest.approx(r.potential_energy, rel=1e-7, abs=1e-12), (ns, name)
