"""The double-coordinate type sets of the boundary against the reference's own GPU code.

The reference instantiates its upward pass and its traversal for three type sets (source_center_gpu.cu:164-170,
upsweep_gpu.cu:134-143, traversal_gpu.cu:635-641): all float, all double ("f64") and double coordinates and centres
with float masses, softenings, multipoles and outputs ("mixed"). For the two double sets this file runs the
reference's TreeBuilder<uint64_t>::update<double>, its upsweep and its traverse (compiled from its sources into
oracle/_ref/libryo_ref_gpu.so) beside this library's steps and traversal on the same tree and groups:

- centres and MAC radii: the reference sums in its centre type, this library in double and rounds once;
- multipoles: float round-off (mixed) or double round-off (f64) of the node's largest moment;
- readBhStats sums and maxima equal;
- accelerations: 1e-9 relative at the 99th percentile for f64 (both sides sum in double with the same
  single-precision rsqrt, only the order and the contraction of the arithmetic differ), 1e-5 for mixed (float
  outputs).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds
from test_gpu_ref_traverse import _ptr, host, ref_fixed_groups, ref_lib, rel_err, sorted_bodies

pytestmark = pytest.mark.gpu


def _ref64_lib():
    lib = ref_lib()
    lib.ref_gpu_build_f64.restype = C.c_int
    lib.ref_gpu_build_f64.argtypes = [C.c_void_p] * 4 + [C.c_size_t, C.c_void_p]
    lib.ref_gpu_upsweep_f64.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_void_p, C.c_void_p, C.c_int]
    lib.ref_gpu_upsweep_mixed.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_void_p, C.c_void_p, C.c_int]
    for name in ("ref_gpu_traverse_f64", "ref_gpu_traverse_mixed"):
        fn = getattr(lib, name)
        fn.restype = C.c_double
        fn.argtypes = ([C.c_uint32] * 3 + [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 15 + [C.c_double, C.c_int] +
                       [C.c_void_p] * 7 + [C.c_int])
    return lib


class RefFlow64:
    """the reference's double build and upsweep of one type set on Hilbert-sorted bodies"""

    def __init__(self, kind, x, y, z, m, h, box, bucket, theta, mdq=False):
        lib = _ref64_lib()
        mt = torch.float64 if kind == "f64" else torch.float32
        d = lambda a, t=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", t)  # noqa: E731
        self.kind, self.mdq = kind, mdq
        self.x, self.y, self.z = d(x), d(y), d(z)
        self.m, self.h = d(m, mt), d(h, mt)
        self.n = len(x)
        self.box = np.ascontiguousarray(box, np.float64)
        torch.cuda.synchronize()
        self.handle = lib.ref_gpu_create(bucket)
        self.num_nodes = lib.ref_gpu_build_f64(self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), self.n,
                                               self.box.ctypes.data_as(C.c_void_p))
        lr, nl = (C.c_int * 23)(), C.c_int(0)
        lib.ref_gpu_tree(self.handle, lr, C.byref(nl))
        self.num_leaves, self.level_range = nl.value, list(lr)
        i32 = lambda k: torch.empty(k, dtype=torch.int32, device="cuda")  # noqa: E731
        self.layout, self.child_offsets = i32(self.num_leaves + 1), i32(self.num_nodes)
        self.leaf_to_internal, self.internal_to_leaf = i32(self.num_leaves), i32(self.num_nodes)
        self.prefixes = torch.empty(self.num_nodes, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        assert lib.ref_gpu_tree_copy(self.handle, _ptr(self.layout), _ptr(self.prefixes), _ptr(self.child_offsets),
                                     _ptr(self.leaf_to_internal), _ptr(self.internal_to_leaf)) == 0
        self.centers = torch.zeros(self.num_nodes, 4, dtype=torch.float64, device="cuda")
        self.multipoles = torch.zeros(self.num_nodes, 12 if mdq else 8, dtype=mt, device="cuda")
        up = lib.ref_gpu_upsweep_f64 if kind == "f64" else lib.ref_gpu_upsweep_mixed
        up(self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.m), self.box.ctypes.data_as(C.c_void_p),
           C.c_float(theta), _ptr(self.centers), _ptr(self.multipoles), int(mdq))
        assert lib.ref_gpu_last_error() == 0

    def close(self):
        ref_lib().ref_gpu_destroy(self.handle)


def ref_traverse64(f, groups, shells=0, boxL=(0.0, 0.0, 0.0), G=1.0):
    lib = _ref64_lib()
    at = torch.float64 if f.kind == "f64" else torch.float32
    p, ax, ay, az = (torch.zeros(f.n, dtype=at, device="cuda") for _ in range(4))
    stats, retries = (C.c_uint64 * 5)(), C.c_uint64(0)
    bl = np.asarray(boxL, np.float64)
    gs, ge = groups[:-1].contiguous(), groups[1:].contiguous()
    fn = lib.ref_gpu_traverse_f64 if f.kind == "f64" else lib.ref_gpu_traverse_mixed
    torch.cuda.synchronize()
    pot = fn(0, f.n, int(gs.numel()), _ptr(gs), _ptr(ge), 1, _ptr(f.x), _ptr(f.y), _ptr(f.z), _ptr(f.m), _ptr(f.h),
             _ptr(f.x), _ptr(f.y), _ptr(f.z), _ptr(f.m), _ptr(f.h), _ptr(f.child_offsets), _ptr(f.internal_to_leaf),
             _ptr(f.layout), _ptr(f.centers), _ptr(f.multipoles), C.c_double(G), shells,
             bl.ctypes.data_as(C.c_void_p), _ptr(p), _ptr(ax), _ptr(ay), _ptr(az), stats, C.byref(retries),
             int(f.mdq))
    assert lib.ref_gpu_last_error() == 0
    return pot, list(stats), p, ax, ay, az


def _bodies(oracle, kind_of_set):
    if kind_of_set == "plummer":
        p = ds.plummer(1 << 16, seed=31, velocities=False)
    else:
        p = ds.uniform_cube(1 << 16, seed=32, eps=0.01)
    # double coordinates that are not float values: a jitter far below the spacing
    rng = np.random.default_rng(33)
    x, y, z = (a.astype(np.float64) + rng.uniform(-1e-9, 1e-9, p.n) for a in (p.x, p.y, p.z))
    # the cube enclosing the jittered bodies (the reference asserts that every body lies in the box)
    lo = np.array([x.min(), y.min(), z.min()])
    ext = float((np.array([x.max(), y.max(), z.max()]) - lo).max()) * (1 + 1e-6)
    box = np.array([lo[0], lo[0] + ext, lo[1], lo[1] + ext, lo[2], lo[2] + ext], np.float64)
    return sorted_bodies(oracle, x, y, z, p.m.astype(np.float64), p.h.astype(np.float64), box) + (box,)


@pytest.mark.parametrize("kind", ["f64", "mixed"])
@pytest.mark.parametrize("mdq", [False, True])
def test_double_upsweep_steps_match_reference(oracle, kind, mdq):
    import ryoanji_b200 as ryo
    x, y, z, m, h, box = _bodies(oracle, "plummer")
    f = RefFlow64(kind, x, y, z, m, h, box, 64, 0.5, mdq=mdq)
    try:
        centers = torch.zeros_like(f.centers)
        mp = torch.zeros_like(f.multipoles)
        ryo.compute_leaf_source_center(f.x, f.y, f.z, f.m, f.leaf_to_internal, f.layout, centers)
        nlev = max(i for i in range(22) if f.level_range[i + 1] > f.level_range[i]) + 1
        ryo.upsweep_centers(nlev, f.level_range, f.child_offsets, centers)
        ryo.compute_leaf_multipoles(f.x, f.y, f.z, f.m, f.leaf_to_internal, f.layout, centers, mp, mdq=mdq)
        for level in range(nlev - 1, 0, -1):
            ryo.upsweep_multipoles(f.level_range[level], f.level_range[level + 1], f.child_offsets, centers, mp,
                                   mdq=mdq)
        b = ryo.Box(*[float(v) for v in box])
        ryo.set_mac(f.prefixes, centers, 2.0, b)
        c, rc = host(centers), host(f.centers)
        scale = np.abs(rc[:, :3]).max()
        assert np.abs(c[:, :3] - rc[:, :3]).max() <= 1e-13 * scale
        assert np.allclose(c[:, 3], rc[:, 3], rtol=1e-12, atol=0)
        q, rq = host(mp).astype(np.float64), host(f.multipoles).astype(np.float64)
        tol = 1e-11 if kind == "f64" else 2e-5  # the reference accumulates float multipoles in float
        big = np.maximum(np.abs(rq[:, 1:]).max(axis=1), np.abs(q[:, 1:]).max(axis=1)) + 1e-300
        assert np.all(np.abs(q[:, 1:] - rq[:, 1:]).max(axis=1) <= tol * big)
        assert np.allclose(q[:, 0], rq[:, 0], rtol=tol, atol=0)
    finally:
        f.close()


@pytest.mark.parametrize("kind", ["f64", "mixed"])
@pytest.mark.parametrize("dataset,mdq", [("plummer", False), ("cube", False), ("plummer", True)])
def test_double_traverse_matches_reference(oracle, kind, dataset, mdq):
    import ryoanji_b200 as ryo
    x, y, z, m, h, box = _bodies(oracle, dataset)
    f = RefFlow64(kind, x, y, z, m, h, box, 64, 0.5, mdq=mdq)
    try:
        groups = torch.from_numpy(ref_fixed_groups(f.n).view(np.int32)).cuda()
        rpot, rst, rp, rax, ray, raz = ref_traverse64(f, groups)
        at = torch.float64 if kind == "f64" else torch.float32
        p, ax, ay, az = (torch.zeros(f.n, dtype=at, device="cuda") for _ in range(4))
        pot, gm, gp = ryo.traverse(groups, 1, f.x, f.y, f.z, f.m, f.h, f.x, f.y, f.z, f.m, f.h, f.child_offsets,
                                   f.internal_to_leaf, f.layout, f.centers, f.multipoles, 1.0, 0, None, p, ax, ay,
                                   az, group_counts=True, mdq=mdq)
        st = ryo.read_bh_stats()
        assert st[:4] == rst[:4], (st, rst)
        e = rel_err(host(ax), host(ay), host(az), host(rax), host(ray), host(raz))
        tol = 1e-9 if kind == "f64" else 1e-5
        assert np.percentile(e, 99) <= tol and e.max() <= 50 * tol, (np.percentile(e, 99), e.max())
        assert abs(pot - rpot) <= 1e-5 * abs(rpot)
    finally:
        f.close()


def test_mixed_traverse_agrees_with_float_traverse(oracle):
    """the mixed instantiation on float-representable inputs equals the float one to float round-off"""
    import ryoanji_b200 as ryo
    p = ds.plummer(1 << 15, seed=34, velocities=False)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float64)
    x, y, z, m, h = sorted_bodies(oracle, p.x.astype(np.float64), p.y.astype(np.float64), p.z.astype(np.float64),
                                  p.m.astype(np.float64), p.h.astype(np.float64), box)
    f = RefFlow64("mixed", x, y, z, m, h, box, 32, 0.5)
    try:
        groups = torch.from_numpy(ref_fixed_groups(f.n).view(np.int32)).cuda()
        out = {}
        for label, cast in (("mixed", lambda t: t), ("f32", lambda t: t.float())):
            acc = [torch.zeros(f.n, device="cuda") for _ in range(4)]
            ryo.traverse(groups, 1, *(cast(t) for t in (f.x, f.y, f.z)), f.m, f.h, *(cast(t) for t in (f.x, f.y, f.z)),
                         f.m, f.h, f.child_offsets, f.internal_to_leaf, f.layout, cast(f.centers), f.multipoles, 1.0,
                         0, None, *acc)
            out[label] = [host(a) for a in acc]
        e = rel_err(*out["f32"][1:], *out["mixed"][1:])
        assert np.percentile(e, 99) < 1e-4
    finally:
        f.close()


def _root_expansion(x, y, z, m):
    """the root's CartesianQuadrupole about its centre of mass (P2M, cartesian_qpole.hpp:67-108), in double"""
    w = np.abs(m)
    c = np.array([np.sum(w * a) / w.sum() for a in (x, y, z)])
    r = [a - ci for a, ci in zip((x, y, z), c)]
    raw = [np.sum(m * r[i] * r[j]) for i, j in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))]
    tr = raw[0] + raw[3] + raw[5]
    q = [m.sum(), 3 * raw[0] - tr, 3 * raw[1], 3 * raw[2], 3 * raw[3] - tr, 3 * raw[4], 3 * raw[5] - tr, tr]
    return c, np.array(q)


@pytest.mark.parametrize("kind", ["f32", "f64", "mixed"])
def test_ewald_matches_reference_gpu(kind):
    """computeGravityEwaldGpu for the three type sets of the reference (ewald.cu:101-110) against the reference's own
    GPU kernel on the same groups: the correction's accelerations and potentials to the round-off of the set (the
    reference sums its reciprocal space in the coordinate type, this library in double), and the energy increment"""
    import ryoanji_b200 as ryo
    lib = ref_lib()
    lib.ref_gpu_ewald.restype = C.c_double
    # kind, root centre, root multipole; first, last, numGroups; gStart, gEnd, x, y, z, m; box6, G; ugrav, ax, ay,
    # az, settings
    lib.ref_gpu_ewald.argtypes = ([C.c_int, C.c_void_p, C.c_void_p] + [C.c_uint32] * 3 + [C.c_void_p] * 6 +
                                  [C.c_void_p, C.c_float] + [C.c_void_p] * 5)
    p = ds.periodic_box(4096, seed=51, eps=0.01)
    rng = np.random.default_rng(52)
    m64 = rng.uniform(0.5, 1.5, p.n) / p.n
    c, q = _root_expansion(p.x.astype(np.float64), p.y.astype(np.float64), p.z.astype(np.float64), m64)
    ct = torch.float32 if kind == "f32" else torch.float64
    mt = torch.float64 if kind == "f64" else torch.float32
    x, y, z = (torch.from_numpy(a).to("cuda", ct) for a in (p.x, p.y, p.z))
    m = torch.from_numpy(m64).to("cuda", mt)
    groups = torch.from_numpy(ref_fixed_groups(p.n).view(np.int32)).cuda()
    gs, ge = groups[:-1].contiguous(), groups[1:].contiguous()
    box6 = np.array([0, 1, 0, 1, 0, 1], np.float64)
    settings = np.array([1, 2.6, 2.8, 2.0, 3.0e-3], np.float64)
    ref = [torch.zeros(p.n, dtype=mt, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    rtot = lib.ref_gpu_ewald({"f32": 0, "f64": 1, "mixed": 2}[kind], c.ctypes.data_as(C.c_void_p),
                             q.ctypes.data_as(C.c_void_p), 0, p.n, int(gs.numel()), _ptr(gs), _ptr(ge), _ptr(x),
                             _ptr(y), _ptr(z), _ptr(m), box6.ctypes.data_as(C.c_void_p), C.c_float(1.0),
                             *[_ptr(t) for t in ref], settings.ctypes.data_as(C.c_void_p))
    assert lib.ref_gpu_last_error() == 0
    ours = [torch.zeros(p.n, dtype=mt, device="cuda") for _ in range(4)]
    box = ryo.Box(0.0, 1.0, 0.0, 1.0, 0.0, 1.0, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    tot = ryo.compute_gravity_ewald(c, q, groups, x, y, z, m, box, 1.0, *ours)
    a_ref = np.stack([host(t).astype(np.float64) for t in ref[1:]])
    a_our = np.stack([host(t).astype(np.float64) for t in ours[1:]])
    scale = np.abs(a_ref).max()
    tol = {"f32": 2e-5, "f64": 1e-9, "mixed": 2e-6}[kind]
    assert np.abs(a_our - a_ref).max() <= tol * scale, (np.abs(a_our - a_ref).max() / scale)
    u_ref, u_our = host(ref[0]).astype(np.float64), host(ours[0]).astype(np.float64)
    assert np.abs(u_our - u_ref).max() <= tol * np.abs(u_ref).max()
    assert abs(tot - rtot) <= 1e-5 * abs(rtot)
