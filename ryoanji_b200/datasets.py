"""Seeded synthetic particle sets for the gravity workloads (numpy, float32 outputs).

- uniform cube in [-1, 1]^3 (or any box), equal masses;
- Plummer sphere: radii by the inverse of the cumulative mass M(r) = r^3 / (r^2 + a^2)^(3/2), i.e.
  r = a / sqrt(U^(-2/3) - 1), redrawn beyond 50 a; isotropic directions; velocities by the rejection method of
  Aarseth, Henon & Wielen (1974): q = v / v_esc with density q^2 (1 - q^2)^(7/2), v_esc = sqrt(2 G M / a) (1 +
  r^2 / a^2)^(-1/4);
- Hernquist halo: r = a sqrt(U) / (1 - sqrt(U)) (inverse of M(r) = r^2 / (r + a)^2), redrawn beyond 20 a;
- clustered set of Hernquist halos with log-uniform masses;
- periodic unit box, uniform.

Softening follows the reference's P2P clamp radius h_i + h_j, so a Plummer-style eps maps to h = eps / 2.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Particles:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    m: np.ndarray
    h: np.ndarray
    vx: np.ndarray | None = None
    vy: np.ndarray | None = None
    vz: np.ndarray | None = None
    box: tuple | None = None  # (x0, x1, y0, y1, z0, z1) when the set defines one
    periodic: bool = False

    @property
    def n(self) -> int:
        return len(self.x)


def _f32(*a):
    return tuple(np.ascontiguousarray(v, dtype=np.float32) for v in a)


def _directions(rng, n):
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t


def uniform_cube(n: int, seed: int = 0, lo: float = -1.0, hi: float = 1.0, eps: float = 0.0,
                 h_zero: float = 1e-6) -> Particles:
    """n bodies i.i.d. uniform in [lo, hi]^3, masses 1/n; eps = 0 uses h = h_zero (see module docstring)"""
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(lo, hi, n) for _ in range(3))
    m = np.full(n, 1.0 / n)
    h = np.full(n, eps / 2 if eps > 0 else h_zero)
    return Particles(*_f32(x, y, z, m, h), box=(lo, hi, lo, hi, lo, hi))


def periodic_box(n: int, seed: int = 0, L: float = 1.0, eps: float = 0.0, h_zero: float = 1e-6) -> Particles:
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(0.0, L, n) for _ in range(3))
    # keep the open upper face out of the box
    x, y, z = (np.minimum(v, np.nextafter(np.float32(L), np.float32(0))) for v in (x, y, z))
    m = np.full(n, 1.0 / n)
    h = np.full(n, eps / 2 if eps > 0 else h_zero)
    p = Particles(*_f32(x, y, z, m, h), box=(0.0, L, 0.0, L, 0.0, L), periodic=True)
    zero = np.zeros(n, np.float32)
    p.vx, p.vy, p.vz = zero.copy(), zero.copy(), zero.copy()
    return p


def plummer(n: int, seed: int = 0, a: float = 1.0, M: float = 1.0, G: float = 1.0, eps: float | None = 0.01,
            rmax: float = 50.0, velocities: bool = True, center=(0.0, 0.0, 0.0)) -> Particles:
    """Plummer sphere of n equal masses; eps defaults to 0.01 a (h = eps / 2)"""
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        u = rng.uniform(0.0, 1.0, todo.size)
        u = np.maximum(u, 1e-300)
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        ok = rr <= rmax * a
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    dx, dy, dz = _directions(rng, n)
    x, y, z = r * dx + center[0], r * dy + center[1], r * dz + center[2]
    m = np.full(n, M / n)
    e = 0.01 * a if eps is None else eps
    h = np.full(n, e / 2)
    p = Particles(*_f32(x, y, z, m, h))
    if velocities:
        q = np.empty(n)
        todo = np.arange(n)
        while todo.size:
            xq = rng.uniform(0.0, 1.0, todo.size)
            yq = rng.uniform(0.0, 0.1, todo.size)
            ok = yq < xq * xq * (1.0 - xq * xq) ** 3.5
            q[todo[ok]] = xq[ok]
            todo = todo[~ok]
        vesc = np.sqrt(2.0 * G * M / a) * (1.0 + (r / a) ** 2) ** -0.25
        v = q * vesc
        ux, uy, uz = _directions(rng, n)
        p.vx, p.vy, p.vz = _f32(v * ux, v * uy, v * uz)
    return p


def hernquist_radii(rng, n, a, rcut=20.0):
    r = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        s = np.sqrt(rng.uniform(0.0, 1.0, todo.size))
        s = np.minimum(s, 1.0 - 1e-12)
        rr = a * s / (1.0 - s)
        ok = rr <= rcut * a
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    return r


def hernquist_halos(n: int, num_halos: int = 64, seed: int = 0, mass_decades: float = 2.0, a_range=(0.01, 0.05),
                    eps: float = 0.0, h_zero: float = 1e-6) -> Particles:
    """clustered set: halos with log-uniform masses over @p mass_decades, centres uniform in [-1, 1]^3, total mass 1"""
    rng = np.random.default_rng(seed)
    w = 10.0 ** rng.uniform(0.0, mass_decades, num_halos)
    w /= w.sum()
    counts = np.floor(w * n).astype(np.int64)
    counts[: n - counts.sum()] += 1
    scale = rng.uniform(a_range[0], a_range[1], num_halos)
    centers = rng.uniform(-1.0, 1.0, (num_halos, 3))
    xs, ys, zs = [], [], []
    for k in range(num_halos):
        c = int(counts[k])
        if c == 0:
            continue
        r = hernquist_radii(rng, c, scale[k])
        dx, dy, dz = _directions(rng, c)
        xs.append(centers[k, 0] + r * dx)
        ys.append(centers[k, 1] + r * dy)
        zs.append(centers[k, 2] + r * dz)
    x, y, z = np.concatenate(xs), np.concatenate(ys), np.concatenate(zs)
    perm = rng.permutation(n)
    m = np.full(n, 1.0 / n)
    h = np.full(n, eps / 2 if eps > 0 else h_zero)
    return Particles(*_f32(x[perm], y[perm], z[perm], m, h))


def gaussian(n: int, seed: int = 0, sigma: float = 0.2, eps: float = 0.0, h_zero: float = 1e-6) -> Particles:
    rng = np.random.default_rng(seed)
    x, y, z = (np.clip(rng.normal(0.0, sigma, n), -1.0, 1.0) for _ in range(3))
    m = rng.uniform(0.5, 1.5, n) / n
    h = np.full(n, eps / 2 if eps > 0 else h_zero)
    return Particles(*_f32(x, y, z, m, h), box=(-1.0, 1.0, -1.0, 1.0, -1.0, 1.0))


def cube_box(p: Particles, pad: float = 0.0):
    """the cube enclosing the set (lower corner at the minimum, side = largest extent)"""
    lo = np.array([p.x.min(), p.y.min(), p.z.min()], np.float64)
    hi = np.array([p.x.max(), p.y.max(), p.z.max()], np.float64)
    ext = float((hi - lo).max()) * (1 + pad)
    return (lo[0], lo[0] + ext, lo[1], lo[1] + ext, lo[2], lo[2] + ext)
