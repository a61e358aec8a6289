"""Served stream (ryo_engine_*): continuous batching must not change any request's result.

Each request is run alone and in a mix of requests that arrive at different engine steps; the final states
must agree within 1e-5 relative. Forces in a batch equal the single-system solve's, so the trajectories
agree to rounding. The leapfrog itself is checked against a float64 numpy KDK integrator on a system the tree
evaluates exactly (one leaf, all P2P). Energy drift, admission under the budget and error statuses are checked too.
"""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _requests():
    import ryoanji_b200 as ryo
    pb = ds.periodic_box(2000, seed=4, eps=0.002)
    pb.vx, pb.vy, pb.vz = (np.random.default_rng(k).normal(0, 0.05, pb.n).astype(np.float32) for k in range(3))
    return [
        dict(tag=1, p=ds.plummer(3000, seed=1), steps=5, box=None),
        dict(tag=2, p=ds.uniform_cube(5000, seed=2, eps=0.004), steps=3, box=None),
        dict(tag=3, p=pb, steps=4, box=ryo.Box(*pb.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)),
        dict(tag=4, p=ds.plummer(10000, seed=3), steps=0, box=None),
        dict(tag=5, p=ds.uniform_cube(1500, seed=5, eps=0.01), steps=7, box=None),
        dict(tag=6, p=ds.plummer(800, seed=6, a=0.3), steps=2, box=None),
    ] + [dict(tag=10 + k, p=ds.plummer(300 + 50 * k, seed=20 + k), steps=1 + k % 3, box=None) for k in range(6)]


def _submit(eng, r, dt=1e-3, out=None):
    p = r["p"]
    eng.submit(r["tag"], p.x, p.y, p.z, p.m, p.h, p.vx, p.vy, p.vz, box=r["box"], steps=r["steps"], dt=dt,
               want_output=True, out=out)


def _drain(eng, max_steps=200):
    res = {}
    for _ in range(max_steps):
        info = eng.step()
        for d in eng.poll():
            res[d["tag"]] = d
        if info["resident"] == 0 and info["queued"] == 0 and info["retired"] == 0:
            break
    return res


def test_each_request_same_alone_and_in_the_mix():
    import ryoanji_b200 as ryo
    reqs = _requests()
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32)
    mix = ryo.Engine(params)
    # staggered arrivals: two at once, then one per step
    _submit(mix, reqs[0])
    _submit(mix, reqs[1])
    mixed = {}
    for r in reqs[2:]:
        mix.step()
        for d in mix.poll():
            mixed[d["tag"]] = d
        _submit(mix, r)
    mixed.update(_drain(mix))
    assert sorted(mixed) == sorted(r["tag"] for r in reqs)
    for r in reqs:
        # alone: arenas reserved up front, final state into a caller's pinned buffer
        alone = ryo.Engine(params, reserve_bodies=20000)
        out = torch.empty((10, r["p"].n), dtype=torch.float32).pin_memory()
        _submit(alone, r, out=out)
        a = _drain(alone)[r["tag"]]
        b = mixed[r["tag"]]
        assert a["steps"] == b["steps"] == r["steps"]
        assert a["state"] is out
        sa, sb = out.numpy(), b["state"]
        scale = np.abs(sa).max(axis=1, keepdims=True) + 1e-30
        rel = float((np.abs(sa - sb) / scale).max())
        assert rel <= 1e-5, (r["tag"], rel)
        assert b["potential"] == pytest.approx(a["potential"], rel=1e-6)
        alone.close()
    mix.close()


def test_leapfrog_matches_float64_reference():
    """50 bodies in one leaf: the tree force is the exact softened sum, so the engine's KDK can be compared with
    a float64 numpy KDK of the same scheme"""
    import ryoanji_b200 as ryo
    p = ds.plummer(50, seed=9)
    K, dt = 20, 2e-3
    eng = ryo.Engine(ryo.SolveParams(theta=0.5, bucket_size=64, group_size=64))
    eng.submit(7, p.x, p.y, p.z, p.m, p.h, p.vx, p.vy, p.vz, steps=K, dt=dt, want_output=True)
    got = _drain(eng)[7]["state"]

    x = np.stack([p.x, p.y, p.z], 1).astype(np.float64)
    v = np.stack([p.vx, p.vy, p.vz], 1).astype(np.float64)
    m = p.m.astype(np.float64)
    h = p.h.astype(np.float64)

    def acc(x):
        d = x[None, :, :] - x[:, None, :]
        r2 = (d * d).sum(-1)
        hh = (h[:, None] + h[None, :]) ** 2
        r2e = np.maximum(r2, hh)
        w = m[None, :] / (r2e * np.sqrt(r2e))
        np.fill_diagonal(w, 0.0)
        return (d * w[:, :, None]).sum(1)

    a = acc(x)
    for _ in range(K):
        v += 0.5 * dt * a
        x += dt * v
        a = acc(x)
        v += 0.5 * dt * a
    ref = np.concatenate([x.T, v.T, a.T], 0)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    rel = np.abs(got[:9] - ref) / scale
    assert float(rel.max()) < 2e-4, float(rel.max())


def test_energy_drift_small():
    import ryoanji_b200 as ryo
    p = ds.plummer(4000, seed=12)
    eng = ryo.Engine(ryo.SolveParams(theta=0.4))
    eng.submit(1, p.x, p.y, p.z, p.m, p.h, p.vx, p.vy, p.vz, steps=30, dt=1e-3)
    d = _drain(eng)[1]
    e1 = d["kinetic"] + d["potential"]
    assert abs(e1 - d["initial"]) / abs(d["initial"]) < 2e-3, (e1, d["initial"])


def test_admission_respects_budget():
    import ryoanji_b200 as ryo
    reqs = [ds.plummer(1000, seed=30 + k) for k in range(6)]
    # 256 B per body: 2.5 requests fit in 640 kB
    eng = ryo.Engine(ryo.SolveParams(), hbm_budget_bytes=640e3, bytes_per_body=256.0)
    for k, p in enumerate(reqs):
        eng.submit(k, p.x, p.y, p.z, p.m, p.h, p.vx, p.vy, p.vz, steps=2, dt=1e-3)
    first = eng.step()
    assert first["resident"] == 2 and first["queued"] == 4
    assert eng.status()["bytes_in_use"] <= 640e3
    done = _drain(eng)
    assert sorted(done) == list(range(6))
    big = ds.plummer(3000, seed=40)
    with pytest.raises(ryo.RyoError):
        eng.submit(99, big.x, big.y, big.z, big.m, big.h, steps=1)
    eng.close()


def test_submit_rejects_bad_periodic_requests():
    """a periodic request the batched solve would refuse (non-cubic box, replica shells outside [0, 4]) is refused at
    submission, and the requests already resident keep running"""
    import ryoanji_b200 as ryo
    eng = ryo.Engine(ryo.SolveParams())
    ok = ds.plummer(500, seed=50)
    eng.submit(1, ok.x, ok.y, ok.z, ok.m, ok.h, ok.vx, ok.vy, ok.vz, steps=2, dt=1e-3)
    eng.step()
    pb = ds.periodic_box(400, seed=51, eps=0.01)
    per = (ryo.BOUNDARY_PERIODIC,) * 3
    lo, hi = pb.box[0], pb.box[1]
    with pytest.raises(ryo.RyoError) as e:
        eng.submit(2, pb.x, pb.y, pb.z, pb.m, pb.h, box=ryo.Box(lo, hi, lo, hi, lo, hi + 0.5, per), steps=1)
    assert e.value.status == ryo._abi.ERR_NOT_CUBIC
    with pytest.raises(ryo.RyoError) as e:
        eng.submit(3, pb.x, pb.y, pb.z, pb.m, pb.h, box=ryo.Box(*pb.box, boundary=per), num_shells=5, steps=1)
    assert e.value.status == ryo._abi.ERR_BAD_ARG
    done = _drain(eng)
    assert sorted(done) == [1]
    eng.close()


def test_capped_steps_keep_results_and_favour_short_requests():
    """with a step cap, each step advances the requests with the least remaining work that fit; the results stay the
    uncapped engine's, the least-work request retires first, and some steps leave requests waiting"""
    import ryoanji_b200 as ryo
    reqs = _requests()
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32)
    capped = ryo.Engine(params, max_step_bodies=4000)
    for r in reqs:
        _submit(capped, r)
    finished, partial_steps = {}, 0
    for step in range(500):
        info = capped.step()
        partial_steps += info["solved"] < info["resident"]
        for d in capped.poll():
            finished[d["tag"]] = (step, d)
        if len(finished) == len(reqs):
            break
    assert len(finished) == len(reqs) and partial_steps > 0
    ref = ryo.Engine(params, max_step_bodies=0)
    for r in reqs:
        _submit(ref, r)
    full = _drain(ref)
    for r in reqs:
        sa, sb = full[r["tag"]]["state"], finished[r["tag"]][1]["state"]
        scale = np.abs(sa).max(axis=1, keepdims=True) + 1e-30
        assert float((np.abs(sa - sb) / scale).max()) <= 1e-5, r["tag"]
    work = {r["tag"]: r["p"].n * (r["steps"] + 1) for r in reqs}
    first = min(finished, key=lambda t: (finished[t][0], work[t]))
    assert work[first] == min(work.values())
    capped.close()
    ref.close()


def test_capped_step_takes_every_request_that_fits_in_priority_order():
    """a capped step goes down the priority order (least remaining work first) and takes each request that still
    fits: a request too large for the cap does not keep the smaller ones behind it out of the step"""
    import ryoanji_b200 as ryo
    params = ryo.SolveParams(theta=0.5, bucket_size=32, group_size=32)
    # remaining work (bodies x force evaluations to come): a 1000 x 3, b 3500 x 1, c 2500 x 5; order a, b, c
    reqs = [dict(tag=1, p=ds.plummer(1000, seed=31), steps=2, box=None),
            dict(tag=2, p=ds.plummer(3500, seed=32), steps=0, box=None),
            dict(tag=3, p=ds.plummer(2500, seed=33), steps=4, box=None)]
    eng = ryo.Engine(params, max_step_bodies=4000)
    for r in reqs:
        _submit(eng, r)
    info = eng.step()
    # a (1000) fits, b (1000 + 3500) does not, c (1000 + 2500) does
    assert info["resident"] == 3 and info["solved"] == 2 and info["residentBodies"] == 7000, info
    done = _drain(eng)
    for d in eng.poll():
        done[d["tag"]] = d
    ref = ryo.Engine(params, max_step_bodies=0)
    for r in reqs:
        _submit(ref, r)
    full = _drain(ref)
    for r in reqs:
        sa, sb = full[r["tag"]]["state"], done[r["tag"]]["state"]
        scale = np.abs(sa).max(axis=1, keepdims=True) + 1e-30
        assert float((np.abs(sa - sb) / scale).max()) <= 1e-5, r["tag"]
    eng.close()
    ref.close()
