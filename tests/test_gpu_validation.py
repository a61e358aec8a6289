"""Settings the reference refuses are refused here with a status, before any work: Ewald with ceil(hCut) > 3
(ryoanji/src/ryoanji/nbody/ewald.hpp:52-60 asserts it; the k-space tables here are sized for it), negative settings
and a zero alpha with Ewald on. Open boxes ignore the Ewald settings, as the reference's open solves do."""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _arrays(p):
    dev = [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    return dev + [torch.empty(p.n, device="cuda") for _ in range(4)]


@pytest.mark.parametrize("settings", [dict(hCut=3.5), dict(hCut=-1.0), dict(lCut=-0.5), dict(alpha_scale=0.0)])
def test_solve_refuses_ewald_settings_the_reference_refuses(settings):
    import ryoanji_b200 as ryo
    p = ds.periodic_box(2000, seed=9, eps=0.01)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    params = ryo.SolveParams(box=box, ewald=ryo.EwaldSettings(**settings))
    with pytest.raises(ryo.RyoError) as e:
        ryo.solve(*_arrays(p), params=params)
    assert e.value.status == ryo._abi.ERR_BAD_ARG and "ewald" in str(e.value)
    # the same settings are not used, hence not checked, for an open box
    params = ryo.SolveParams(ewald=ryo.EwaldSettings(**settings))
    ryo.solve(*_arrays(ds.uniform_cube(2000, seed=10, eps=0.01)), params=params)


def test_ewald_at_the_limit_still_runs():
    """hCut = 3 (ceil 3) is the largest the reference accepts"""
    import ryoanji_b200 as ryo
    p = ds.periodic_box(2000, seed=11, eps=0.01)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    arrays = _arrays(p)
    ryo.solve(*arrays, params=ryo.SolveParams(box=box, ewald=ryo.EwaldSettings(hCut=3.0)))
    assert all(bool(torch.isfinite(a).all()) for a in arrays[5:])


def test_engine_and_particle_ewald_refuse_them_too():
    """the engine applies its Ewald settings to periodic requests only, as the single-system solve does: creation
    and open requests accept them, a periodic submission is refused"""
    import ryoanji_b200 as ryo
    bad = ryo.EwaldSettings(hCut=3.5)
    eng = ryo.Engine(ryo.SolveParams(ewald=bad))
    try:
        q = ds.uniform_cube(300, seed=13, eps=0.01)
        zero = np.zeros(q.n, np.float32)
        eng.submit(1, *(torch.from_numpy(a) for a in (q.x, q.y, q.z, q.m, q.h, zero, zero, zero)), steps=1,
                   dt=1e-3)
        pb = ds.periodic_box(300, seed=14, eps=0.01)
        box = ryo.Box(*pb.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
        with pytest.raises(ryo.RyoError) as e:
            eng.submit(2, *(torch.from_numpy(a) for a in (pb.x, pb.y, pb.z, pb.m, pb.h, zero, zero, zero)),
                       box=box, steps=1, dt=1e-3)
        assert e.value.status == ryo._abi.ERR_BAD_ARG and "ewald" in str(e.value).lower()
        while eng.status()["queued"] or eng.status()["resident"]:
            eng.step()
        assert [d["tag"] for d in eng.poll()] == [1]
    finally:
        eng.close()
    p = ds.periodic_box(500, seed=12, eps=0.01)
    dev = [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    targets = torch.arange(0, 500, 50, dtype=torch.int64, device="cuda")
    with pytest.raises(ryo.RyoError) as e:
        ryo.ewald_targets_f64(targets, *dev, L=1.0, ewald=bad)
    assert e.value.status == ryo._abi.ERR_BAD_ARG
    np.testing.assert_equal(p.n, 500)


@pytest.mark.parametrize("shells", [-1, 5])
def test_solve_refuses_replica_shells_outside_0_4(shells):
    """a negative count would traverse nothing and return zero forces; the batched solve and the engine refuse the
    same range"""
    import ryoanji_b200 as ryo
    p = ds.periodic_box(1000, seed=15, eps=0.01)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    with pytest.raises(ryo.RyoError) as e:
        ryo.solve(*_arrays(p), params=ryo.SolveParams(box=box, num_shells=shells))
    assert e.value.status == ryo._abi.ERR_BAD_ARG and "numShells" in str(e.value)


def _tiny_tree():
    import ryoanji_b200 as ryo
    p = ds.uniform_cube(512, seed=16, eps=0.01)
    x, y, z, m, h = (torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h))
    tb = ryo.TreeBuilder(16)
    box = ryo.Box(-1.0, 1.0, -1.0, 1.0, -1.0, 1.0)
    nn = tb.update(x, y, z, box)
    centers = torch.zeros(nn, 4, device="cuda")
    mp = torch.zeros(nn, 8, device="cuda")
    return tb, box, (x, y, z, m, h), centers, mp


@pytest.mark.parametrize("kind", ["empty", "over_64", "before_first", "past_last"])
def test_traverse_refuses_bad_caller_groups(kind):
    """every caller group must hold 1 to 64 targets inside [firstBody, lastBody)"""
    import ryoanji_b200 as ryo
    tb, box, (x, y, z, m, h), centers, mp = _tiny_tree()
    g = {"empty": [0, 64, 64, 128], "over_64": [0, 65, 128], "before_first": [0, 64, 128],
         "past_last": [448, 512, 576]}[kind]
    groups = torch.tensor(g, dtype=torch.int32, device="cuda")
    first = 64 if kind == "before_first" else 0
    last = 512 if kind != "past_last" else 512
    p, ax, ay, az = (torch.zeros(x.numel(), device="cuda") for _ in range(4))
    with pytest.raises(ryo.RyoError) as e:
        ryo.traverse(groups, 1, x, y, z, m, h, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(), tb.layout(),
                     centers, mp, 1.0, 0, None, p, ax, ay, az, first_body=first, last_body=last)
    assert e.value.status == ryo._abi.ERR_BAD_ARG


@pytest.mark.parametrize("bad", [-1, 500])
def test_direct_targets_refuse_an_index_outside_the_bodies(bad):
    import ryoanji_b200 as ryo
    p = ds.uniform_cube(500, seed=17, eps=0.01)
    dev = [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    targets = torch.tensor([0, 7, bad], dtype=torch.int64, device="cuda")
    with pytest.raises(ryo.RyoError) as e:
        ryo.direct_targets_f64(targets, *dev)
    assert e.value.status == ryo._abi.ERR_BAD_ARG


def test_bounding_box_is_the_exact_min_and_max():
    """ryo_compute_bounding_box_f32: exact FP64 minimum and maximum of every axis (no rounding: float inputs)"""
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(18)
    for n in (1, 7, 1000, 1 << 20):
        xyz = [rng.standard_normal(n).astype(np.float32) * s for s in (1.0, 1e-3, 1e4)]
        if n > 8:
            xyz[0][n // 3] = np.float32(-3.5e7)
            xyz[2][-1] = np.float32(np.nextafter(np.float32(9e5), np.float32(1e9)))
        b = ryo.compute_bounding_box(*(torch.from_numpy(a).cuda() for a in xyz))
        want = [v for a in xyz for v in (float(a.min()), float(a.max()))]
        assert list(b) == want, (n, list(b), want)


def test_sort_look_back_wait_runs_out_and_reports():
    """the onesweep look-back's bounded wait: a tile whose predecessor never publishes gives up after its poll limit,
    raises the flag the host reads (RYO_ERR_TIMEOUT), and leaves the context usable for the next sort"""
    import ryoanji_b200 as ryo
    torch.cuda.synchronize()
    status = ryo.lib.ryo_sort_wait_timeout_selftest(None)
    msg = (ryo.lib.ryo_ctx_last_error(None) or b"").decode()
    assert status == ryo._abi.ERR_TIMEOUT and "timed out" in msg, (status, msg)
    rng = np.random.default_rng(19)
    keys = torch.from_numpy(rng.integers(0, 2**63, 100003, dtype=np.int64)).cuda()
    vals = torch.arange(keys.numel(), dtype=torch.int32, device="cuda")
    want = np.argsort(keys.cpu().numpy(), kind="stable")
    ryo.sort_by_key(keys, vals)
    assert np.array_equal(vals.cpu().numpy(), want)
