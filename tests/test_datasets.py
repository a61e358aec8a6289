"""The seeded workloads of the bench and the tests follow their stated distributions (CPU; the device generators run
on the CPU device here).

Plummer sphere (a = 1, truncated at 50 a): half-mass radius 1.3045 a and virial ratio 2T/|W| = 1 for the
Aarseth-Henon-Wielen velocities. Hernquist radii truncated at 20 a: median 2.062 a. Uniform and periodic sets stay in
their boxes (the periodic ones off the open upper face); the ensemble and the served mix have the stated ranges.
"""
import numpy as np
import torch

from ryoanji_b200 import datasets as ds

PLUMMER_HALF_MASS = 1.3045  # r^3 / (r^2 + 1)^1.5 = M(50) / 2
HERNQUIST_MEDIAN = 2.062    # r^2 / (r + 1)^2 = M(20) / 2


def _virial_ratio(x, y, z, m, vx, vy, vz):
    p = np.stack([x, y, z], 1).astype(np.float64)
    m = np.asarray(m, np.float64)
    t = 0.5 * np.sum(m * (np.asarray(vx, np.float64) ** 2 + np.asarray(vy, np.float64) ** 2 +
                          np.asarray(vz, np.float64) ** 2))
    w = 0.0
    for i in range(0, len(m), 512):
        d = np.linalg.norm(p[i:i + 512, None, :] - p[None, :, :], axis=2)
        mm = m[i:i + 512, None] * m[None, :]
        w -= 0.5 * np.sum(np.divide(mm, d, out=np.zeros_like(d), where=d > 0))
    return 2.0 * t / abs(w)


def test_plummer_half_mass_radius_and_virial_ratio():
    p = ds.plummer(200000, seed=1, velocities=False)
    r = np.sqrt(p.x.astype(np.float64) ** 2 + p.y ** 2 + p.z ** 2)
    assert abs(np.median(r) / PLUMMER_HALF_MASS - 1) < 0.02 and r.max() <= 50.0
    assert np.allclose(p.m.sum(), 1.0, rtol=1e-5) and np.all(p.h == np.float32(0.005))
    q = ds.plummer(3000, seed=2)
    assert abs(_virial_ratio(q.x, q.y, q.z, q.m, q.vx, q.vy, q.vz) - 1.0) < 0.1


def test_device_plummer_matches_the_same_distribution():
    gen = torch.Generator()
    gen.manual_seed(3)
    x, y, z, vx, vy, vz = ds.plummer_device(torch.ones(200000, dtype=torch.float64), gen)
    r = torch.sqrt(x * x + y * y + z * z).numpy()
    assert abs(np.median(r) / PLUMMER_HALF_MASS - 1) < 0.02 and r.max() <= 50.0
    gen.manual_seed(4)
    x, y, z, vx, vy, vz = (t.numpy() for t in ds.plummer_device(torch.ones(3000, dtype=torch.float64), gen))
    assert abs(_virial_ratio(x, y, z, np.full(3000, 1 / 3000), vx, vy, vz) - 1.0) < 0.1


def test_hernquist_radii_median():
    r = ds.hernquist_radii(np.random.default_rng(0), 200000, 1.0)
    assert abs(np.median(r) / HERNQUIST_MEDIAN - 1) < 0.02 and r.max() <= 20.0


def test_boxes_hold_their_bodies():
    c = ds.uniform_cube(10000, seed=5)
    for a in (c.x, c.y, c.z):
        assert a.min() >= -1 and a.max() <= 1
    pb = ds.periodic_box(10000, seed=6)
    for a in (pb.x, pb.y, pb.z):
        assert a.min() >= 0 and a.max() < 1
    q = dict(tag=0, n=20000, kind="periodic", steps=1, dt=1e-3, arrival=0.0, seed=7)
    for a in ds.request_bodies(q, device="cpu")[:3]:
        assert float(a.min()) >= 0 and float(a.max()) < 1


def test_ensemble_and_served_mix_ranges():
    sizes, radii = ds.ensemble_sizes(1024, seed=0)
    assert sizes.min() >= 2 ** 10 and sizes.max() <= 2 ** 18 and 0.5 <= radii.min() and radii.max() <= 2.0
    x, y, z, m, h, vx, vy, vz = ds.plummer_ensemble(sizes[:4], radii[:4], device="cpu")
    assert len(x) == int(sizes[:4].sum()) and all(t.dtype == torch.float32 for t in (x, m, h))
    first = np.concatenate([[0], np.cumsum(sizes[:4])])
    for k in range(4):  # each system has mass 1 and softening 0.005 a
        assert abs(float(m[first[k]:first[k + 1]].double().sum()) - 1.0) < 1e-5
        assert np.allclose(h[first[k]:first[k + 1]].numpy(), 0.005 * radii[k], rtol=1e-6)
    reqs = ds.served_requests(2000, seed=1, rate_per_s=24.0)
    t = np.array([q["arrival"] for q in reqs])
    assert t[0] == 0 and np.all(np.diff(t) >= 0) and abs(np.mean(np.diff(t)) * 24.0 - 1) < 0.1
    assert all(1 <= q["steps"] <= 64 and 2 ** 12 <= q["n"] <= 2 ** 22 for q in reqs)
    kinds = [q["kind"] for q in reqs]
    assert abs(kinds.count("periodic") / len(kinds) - 0.10) < 0.03
