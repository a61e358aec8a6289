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


# ------------------------------------------------------------------------------------------------------------------
# device-side generators for the batched ensemble and the served stream (torch, seeded generator on the device)

def _t_directions(n, gen, device):
    import torch
    cos_t = torch.rand(n, generator=gen, device=device, dtype=torch.float64) * 2 - 1
    phi = torch.rand(n, generator=gen, device=device, dtype=torch.float64) * (2 * np.pi)
    sin_t = torch.sqrt(1 - cos_t * cos_t)
    return sin_t * torch.cos(phi), sin_t * torch.sin(phi), cos_t


def plummer_device(a, gen, G: float = 1.0, total_mass=None, rmax: float = 50.0, velocities: bool = True):
    """Plummer bodies with per-body scale radius a (torch float64 tensor on the device; systems are runs of equal
    a): r = a / sqrt(U^(-2/3) - 1) resampled above rmax a, isotropic directions, Aarseth-Henon-Wielen velocities
    for a system of mass total_mass (per body, default 1). Returns float64 tensors (x, y, z, vx, vy, vz)."""
    import torch
    n, device = a.numel(), a.device
    M = torch.ones_like(a) if total_mass is None else total_mass
    r = torch.empty(n, dtype=torch.float64, device=device)
    todo = torch.arange(n, device=device)
    while todo.numel():
        u = torch.rand(todo.numel(), generator=gen, device=device, dtype=torch.float64).clamp_min(1e-300)
        rr = a[todo] / torch.sqrt(u ** (-2.0 / 3.0) - 1.0)
        ok = rr <= rmax * a[todo]
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    dx, dy, dz = _t_directions(n, gen, device)
    if not velocities:
        z = torch.zeros_like(r)
        return r * dx, r * dy, r * dz, z, z.clone(), z.clone()
    q = torch.empty(n, dtype=torch.float64, device=device)
    todo = torch.arange(n, device=device)
    while todo.numel():
        xq = torch.rand(todo.numel(), generator=gen, device=device, dtype=torch.float64)
        yq = torch.rand(todo.numel(), generator=gen, device=device, dtype=torch.float64) * 0.1
        ok = yq < xq * xq * (1 - xq * xq) ** 3.5
        q[todo[ok]] = xq[ok]
        todo = todo[~ok]
    vesc = torch.sqrt(2 * G * M / a) * (1 + (r / a) ** 2) ** -0.25
    v = q * vesc
    ux, uy, uz = _t_directions(n, gen, device)
    return r * dx, r * dy, r * dz, v * ux, v * uy, v * uz


def ensemble_sizes(num_systems: int = 1024, seed: int = 0, lo_log2: float = 10.0, hi_log2: float = 18.0):
    """system sizes round(2^U[lo, hi]) and Plummer scale radii U[0.5, 2] of the batched ensemble"""
    rng = np.random.default_rng(seed)
    sizes = np.rint(2.0 ** rng.uniform(lo_log2, hi_log2, num_systems)).astype(np.int64)
    radii = rng.uniform(0.5, 2.0, num_systems)
    return sizes, radii


def plummer_ensemble(sizes, radii, seed: int = 0, device="cuda"):
    """the concatenated bodies of independent Plummer systems (mass 1, softening eps = 0.01 a, h = eps / 2):
    float32 device tensors x, y, z, m, h, vx, vy, vz"""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    sizes_t = torch.as_tensor(np.asarray(sizes), device=device)
    a = torch.repeat_interleave(torch.as_tensor(np.asarray(radii), dtype=torch.float64, device=device), sizes_t)
    x, y, z, vx, vy, vz = plummer_device(a, gen)
    m = torch.repeat_interleave(1.0 / sizes_t.double(), sizes_t)
    h = 0.005 * a
    return [t.float().contiguous() for t in (x, y, z, m, h, vx, vy, vz)]


def served_requests(num_requests: int, seed: int = 0, rate_per_s: float = 24.0, lo_log2: float = 12.0,
                    hi_log2: float = 22.0):
    """the served-stream request mix: open-loop Poisson arrivals, N = round(2^U[lo, hi]); 45% Plummer (a = 1,
    eps = 0.01, AHW velocities), 45% uniform cube [-1, 1]^3 at rest (h = 1e-6), 10% periodic unit box at rest with
    Ewald (h = 1e-6); K ~ U{1..64} leapfrog steps, dt = 1e-3. Returns descriptions without bodies."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, num_requests))
    out = []
    for k in range(num_requests):
        u = rng.uniform()
        kind = "plummer" if u < 0.45 else ("cube" if u < 0.90 else "periodic")
        out.append(dict(tag=k, n=int(np.rint(2.0 ** rng.uniform(lo_log2, hi_log2))), kind=kind,
                        steps=int(rng.integers(1, 65)), dt=1e-3, arrival=float(t[k]) - float(t[0]),
                        seed=int(rng.integers(1 << 31))))
    return out


def request_bodies(req: dict, device="cuda"):
    """float32 device tensors x, y, z, m, h, vx, vy, vz of one served request"""
    import torch
    n = req["n"]
    gen = torch.Generator(device=device)
    gen.manual_seed(req["seed"])
    if req["kind"] == "plummer":
        x, y, z, vx, vy, vz = plummer_device(torch.ones(n, dtype=torch.float64, device=device), gen)
        h = torch.full((n,), 0.005, dtype=torch.float64, device=device)
    else:
        lo, hi = (-1.0, 1.0) if req["kind"] == "cube" else (0.0, 1.0)
        x, y, z = (torch.rand(n, generator=gen, device=device, dtype=torch.float64) * (hi - lo) + lo
                   for _ in range(3))
        if req["kind"] == "periodic":
            top = float(np.nextafter(np.float32(hi), np.float32(0)))
            x, y, z = (v.clamp_max(top) for v in (x, y, z))
        vx = vy = vz = torch.zeros(n, dtype=torch.float64, device=device)
        h = torch.full((n,), 1e-6, dtype=torch.float64, device=device)
    m = torch.full((n,), 1.0 / n, dtype=torch.float64, device=device)
    return [t.float().contiguous() for t in (x, y, z, m, h, vx, vy, vz)]
