"""The traversal against the reference's own GPU `traverse`, run on the same device.

The reference's plain GPU path (TreeBuilder, the demo's upsweep, computeFixedGroups, traverse and readBhStats;
ryoanji/test/demo.cu:82-104, :171-190) is compiled from the reference sources into oracle/_ref/libryo_ref_gpu.so when
the reference tree was present at build time (oracle/Makefile, target refgpu). Here both traversals read the same
tree, centres, multipoles and 64-body groups, all produced by the reference's own GPU code:

- the interaction statistics of readBhStats (ryoanji/src/ryoanji/nbody/traversal_gpu.cu:686-700): sumP2P, maxP2P,
  sumM2P and maxM2P must be equal (the stack depth is not compared: the reference keeps a breadth-first ring buffer
  in global memory, this library a depth-first stack in shared memory);
- accelerations within 1e-5 relative at the 99th percentile (only the summation order differs: the reference adds
  in its queue order without compensation, this library in batches with Kahan compensation), potentials likewise;
- the total potential within 1e-5 (the reference sums it with float atomics).

When the statistics differ, the test bisects the groups by running the reference on sub-ranges and reports the first
groups whose counts differ, with their counts on both sides.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from conftest import ROOT, golden_cases
from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu

REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libryo_ref_gpu.so")
_LIB = None


def ref_lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(REF_GPU):
            pytest.skip("the reference's GPU path was not built (no reference tree at build time)")
        lib = C.CDLL(REF_GPU)
        lib.ref_gpu_create.restype = C.c_void_p
        lib.ref_gpu_destroy.argtypes = [C.c_void_p]
        lib.ref_gpu_build_f32.restype = C.c_int
        lib.ref_gpu_build_f32.argtypes = [C.c_void_p] + [C.c_void_p] * 3 + [C.c_size_t, C.c_void_p]
        lib.ref_gpu_tree.argtypes = [C.c_void_p] * 3
        lib.ref_gpu_tree_copy.argtypes = [C.c_void_p] * 6
        lib.ref_gpu_upsweep_f32.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_void_p, C.c_void_p, C.c_int]
        lib.ref_gpu_fixed_groups.restype = C.c_long
        lib.ref_gpu_fixed_groups.argtypes = [C.c_uint32, C.c_uint32, C.c_uint, C.c_void_p, C.c_long]
        lib.ref_gpu_traverse_f32.restype = C.c_double
        lib.ref_gpu_traverse_f32.argtypes = ([C.c_uint32] * 3 + [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 15 +
                                             [C.c_float, C.c_int] + [C.c_void_p] * 7 + [C.c_int])
        lib.ref_gpu_last_error.restype = C.c_int
        _LIB = lib
    return _LIB


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def host(t):
    return t.detach().cpu().numpy()


class RefFlow:
    """the reference's build and upsweep on sorted bodies; holds the reference's tree arrays (device)"""

    def __init__(self, x, y, z, m, h, box, bucket, theta, mdq=False):
        lib = ref_lib()
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        self.x, self.y, self.z, self.m, self.h = (d(a) for a in (x, y, z, m, h))
        self.n = len(x)
        self.box = np.ascontiguousarray(box, np.float32)
        torch.cuda.synchronize()
        self.handle = lib.ref_gpu_create(bucket)
        self.num_nodes = lib.ref_gpu_build_f32(self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), self.n,
                                               self.box.ctypes.data_as(C.c_void_p))
        lr = (C.c_int * 23)()
        nl = C.c_int(0)
        lib.ref_gpu_tree(self.handle, lr, C.byref(nl))
        self.num_leaves = nl.value
        self.level_range = list(lr)
        self.layout = torch.empty(self.num_leaves + 1, dtype=torch.int32, device="cuda")
        self.prefixes = torch.empty(self.num_nodes, dtype=torch.int64, device="cuda")
        self.child_offsets = torch.empty(self.num_nodes, dtype=torch.int32, device="cuda")
        self.internal_to_leaf = torch.empty(self.num_nodes, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert lib.ref_gpu_tree_copy(self.handle, _ptr(self.layout), _ptr(self.prefixes), _ptr(self.child_offsets),
                                     None, _ptr(self.internal_to_leaf)) == 0
        self.mdq = mdq
        self.centers = torch.zeros(self.num_nodes, 4, device="cuda")
        self.multipoles = torch.zeros(self.num_nodes, 12 if mdq else 8, device="cuda")
        lib.ref_gpu_upsweep_f32(self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.m),
                                self.box.ctypes.data_as(C.c_void_p), C.c_float(theta), _ptr(self.centers),
                                _ptr(self.multipoles), int(mdq))
        assert lib.ref_gpu_last_error() == 0

    def close(self):
        ref_lib().ref_gpu_destroy(self.handle)


def ref_fixed_groups(n, size=64):
    lib = ref_lib()
    out = np.zeros(n // size + 3, np.uint32)
    ng = lib.ref_gpu_fixed_groups(0, n, size, out.ctypes.data_as(C.c_void_p), len(out))
    return out[:ng + 1]


def ref_traverse(f: RefFlow, gstart, gend, shells=0, boxL=(0.0, 0.0, 0.0), G=1.0):
    """the reference's traverse over the groups [gstart, gend) (device uint32 tensors); returns
    (potential, stats5, retries, p, ax, ay, az)"""
    lib = ref_lib()
    n = f.n
    p, ax, ay, az = (torch.zeros(n, device="cuda") for _ in range(4))
    stats = (C.c_uint64 * 5)()
    retries = C.c_uint64(0)
    bl = np.asarray(boxL, np.float32)
    torch.cuda.synchronize()
    pot = lib.ref_gpu_traverse_f32(0, n, int(gstart.numel()), _ptr(gstart), _ptr(gend), 1, _ptr(f.x), _ptr(f.y),
                                   _ptr(f.z), _ptr(f.m), _ptr(f.h), _ptr(f.x), _ptr(f.y), _ptr(f.z), _ptr(f.m),
                                   _ptr(f.h), _ptr(f.child_offsets), _ptr(f.internal_to_leaf), _ptr(f.layout),
                                   _ptr(f.centers), _ptr(f.multipoles), C.c_float(G), shells,
                                   bl.ctypes.data_as(C.c_void_p), _ptr(p), _ptr(ax), _ptr(ay), _ptr(az), stats,
                                   C.byref(retries), int(f.mdq))
    assert lib.ref_gpu_last_error() == 0
    return pot, list(stats), retries.value, p, ax, ay, az


def our_traverse(f: RefFlow, groups, shells=0, boxL=(0.0, 0.0, 0.0), G=1.0, ctx=None):
    import ryoanji_b200 as ryo
    n = f.n
    p, ax, ay, az = (torch.zeros(n, device="cuda") for _ in range(4))
    pot, gm, gp = ryo.traverse(groups, 1, f.x, f.y, f.z, f.m, f.h, f.x, f.y, f.z, f.m, f.h, f.child_offsets,
                               f.internal_to_leaf, f.layout, f.centers, f.multipoles, G, shells,
                               boxL if shells else None, p, ax, ay, az, ctx=ctx, group_counts=True, mdq=f.mdq)
    stats = ryo.read_bh_stats(ctx)
    return pot, stats, host(gm).view(np.uint32), host(gp).view(np.uint32), p, ax, ay, az


def first_differing_groups(f, gstart, gend, ours_m2p, ours_p2p, shells, boxL, limit=4):
    """bisect the group range with the reference's sums until single groups whose counts differ are found"""
    found = []
    sizes = host(gend).astype(np.int64) - host(gstart).astype(np.int64)

    def sums(lo, hi):
        _, st, _, *_ = ref_traverse(f, gstart[lo:hi], gend[lo:hi], shells, boxL)
        return st[0], st[2]

    def ours(lo, hi):
        return (int((ours_p2p[lo:hi].astype(np.int64) * sizes[lo:hi]).sum()),
                int((ours_m2p[lo:hi].astype(np.int64) * sizes[lo:hi]).sum()))

    stack = [(0, int(gstart.numel()))]
    while stack and len(found) < limit:
        lo, hi = stack.pop()
        if sums(lo, hi) == ours(lo, hi):
            continue
        if hi - lo == 1:
            rp, rm = sums(lo, hi)
            found.append(dict(group=lo, size=int(sizes[lo]), ref_p2p=rp // sizes[lo], ref_m2p=rm // sizes[lo],
                              our_p2p=int(ours_p2p[lo]), our_m2p=int(ours_m2p[lo])))
            continue
        mid = (lo + hi) // 2
        stack += [(mid, hi), (lo, mid)]
    return found


def rel_err(ax, ay, az, rx, ry, rz):
    num = np.sqrt((ax - rx) ** 2 + (ay - ry) ** 2 + (az - rz) ** 2)
    den = np.sqrt(rx.astype(np.float64) ** 2 + ry.astype(np.float64) ** 2 + rz.astype(np.float64) ** 2)
    return num / np.maximum(den, 1e-300)


def sorted_bodies(oracle, x, y, z, m, h, box):
    """bodies in the Hilbert order of the box (the reference sorts only x, y, z; m and h follow here)"""
    keys = oracle.sfc_keys(x, y, z, np.asarray(box, np.float32))
    _, order = oracle.sort_keys(keys)
    return tuple(np.ascontiguousarray(a[order]) for a in (x, y, z, m, h))


def compare(oracle, x, y, z, m, h, box, bucket=64, theta=0.5, shells=0, mdq=False, force_tol=1e-5, rms_norm=False):
    """both traversals on the same tree; with rms_norm the force and potential differences are measured against the
    rms of the reference's field instead of each target's own: in a periodic box without its Ewald correction, and
    with masses of both signs, a target's net field is a small difference of large terms, so a summation-order
    difference far below the terms' round-off is a large fraction of it"""
    xs, ys, zs, ms, hs = sorted_bodies(oracle, x, y, z, m, h, box)
    f = RefFlow(xs, ys, zs, ms, hs, box, bucket, theta, mdq=mdq)
    try:
        g = ref_fixed_groups(f.n)
        groups = torch.from_numpy(g.view(np.int32)).cuda()
        gstart, gend = groups[:-1].contiguous(), groups[1:].contiguous()
        boxL = tuple(float(v) for v in (box[1] - box[0], box[3] - box[2], box[5] - box[4]))
        rpot, rst, rretry, rp, rax, ray, raz = ref_traverse(f, gstart, gend, shells, boxL)
        opot, ost, om2p, op2p, p, ax, ay, az = our_traverse(f, groups, shells, boxL)
        if rst[:4] != ost[:4]:
            diff = first_differing_groups(f, gstart, gend, om2p, op2p, shells, boxL)
            pytest.fail(f"readBhStats differ: reference {rst[:4]} ours {ost[:4]}; first groups: {diff}")
        e = rel_err(host(ax), host(ay), host(az), host(rax), host(ray), host(raz))
        ep = np.abs(host(p) - host(rp)) / np.maximum(np.abs(host(rp)), 1e-30)
        if rms_norm:
            ra = np.stack([host(rax), host(ray), host(raz)]).astype(np.float64)
            oa = np.stack([host(ax), host(ay), host(az)]).astype(np.float64)
            e = np.linalg.norm(oa - ra, axis=0) / np.sqrt((ra * ra).sum(0).mean())
            rpv = host(rp).astype(np.float64)
            ep = np.abs(host(p) - rpv) / np.sqrt((rpv * rpv).mean())
        assert np.percentile(e, 99) <= force_tol, (np.percentile(e, 99), e.max())
        assert e.max() <= 50 * force_tol, e.max()
        assert np.percentile(ep, 99) <= force_tol, np.percentile(ep, 99)
        # the total against the sum of its terms' magnitudes where the terms cancel, else against itself
        scale = 0.5 * float(np.abs(host(rp).astype(np.float64)).sum()) if rms_norm else abs(rpot)
        assert abs(opot - rpot) <= 1e-5 * scale, (opot, rpot)
        return dict(stats=ost, ref_stats=rst, err_p99=float(np.percentile(e, 99)), err_max=float(e.max()),
                    retries=rretry)
    finally:
        f.close()


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_golden_cases_match_reference_gpu(oracle, path):
    c = dict(np.load(path))
    periodic = "ewald_u" in c
    box = c["box"]
    compare(oracle, c["x"], c["y"], c["z"], c["m"], c["h"], box, bucket=int(c["bucket"]), theta=float(c["theta"]),
            shells=1 if periodic else 0, rms_norm=periodic)


def test_uniform_cube_2e18_matches_reference_gpu(oracle):
    p = ds.uniform_cube(1 << 18, seed=11)  # eps = 0 as h = 1e-6: the reference's P2P needs h > 0 for i == j
    r = compare(oracle, p.x, p.y, p.z, p.m, p.h, np.array(p.box, np.float32))
    assert r["stats"][0] > 0 and r["stats"][2] > 0


def test_plummer_2e18_matches_reference_gpu(oracle):
    p = ds.plummer(1 << 18, seed=12, velocities=False)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    compare(oracle, p.x, p.y, p.z, p.m, p.h, box)


def test_plummer_theta_0_3_matches_reference_gpu(oracle):
    p = ds.plummer(1 << 16, seed=13, velocities=False)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    compare(oracle, p.x, p.y, p.z, p.m, p.h, box, theta=0.3, bucket=32)


def test_signed_masses_mdq_match_reference_gpu(oracle):
    """the MDQpole instantiation with signed masses (the isRemote rule keys on the MAC radius, not the mass)"""
    p = ds.gaussian(1 << 15, seed=14)
    rng = np.random.default_rng(14)
    m = (rng.choice([-1.0, 1.0], len(p.x)) / len(p.x)).astype(np.float32)
    h = np.full_like(p.x, 1e-3)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    compare(oracle, p.x, p.y, p.z, m, h, box, theta=0.3, mdq=True, rms_norm=True)


def test_varied_softening_and_masses_match_reference_gpu(oracle):
    """every body its own softening and mass: the general direct sums (the per-pair softening floor (h_i + h_j)^2 and
    the per-source mass) instead of the one-softening and one-mass forms"""
    p = ds.gaussian(1 << 16, seed=21, sigma=0.3)
    rng = np.random.default_rng(21)
    m = (rng.uniform(0.2, 1.8, len(p.x)) / len(p.x)).astype(np.float32)
    h = rng.uniform(1e-4, 1e-2, len(p.x)).astype(np.float32)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    compare(oracle, p.x, p.y, p.z, m, h, box)


def test_clustered_halos_theta_0_7_bucket_16_match_reference_gpu(oracle):
    """a clustered set at a coarse opening angle and small leaves: many approximated cells and many small leaves per
    group"""
    p = ds.hernquist_halos(1 << 17, num_halos=16, seed=22, eps=1e-3)
    box = np.array(ds.cube_box(p, pad=1e-6), np.float32)
    compare(oracle, p.x, p.y, p.z, p.m, p.h, box, theta=0.7, bucket=16)


def test_ragged_small_set_matches_reference_gpu(oracle):
    """fewer bodies than one group of 64 plus a ragged tail: a tree of a few leaves and a partial last group"""
    p = ds.uniform_cube(100, seed=23, eps=1e-3)
    compare(oracle, p.x, p.y, p.z, p.m, p.h, np.array(p.box, np.float32), bucket=8)


def test_periodic_replicas_of_a_cluster_match_reference_gpu(oracle):
    """one shell of periodic replicas (27 images per group) without the Ewald correction, on a cluster inside the unit
    box: its field does not cancel, so each target's own field is the scale (in a uniform box the net field is a small
    remainder of the images' terms). The interaction counts must be equal. The forces differ by more than in an open
    box: the reference moves its targets into each image and back (traversal_gpu.cu:484-505), which leaves residues
    of about one float ulp of the coordinates in the later images, where this library adds each image's shift to the
    original positions. Near the softening length (h = 1e-3) such a residue is about 6e-5 of the force."""
    p = ds.gaussian(1 << 15, seed=24, sigma=0.1, eps=2e-3)
    x, y, z = (np.mod(a + 0.5, 1.0).astype(np.float32) for a in (p.x, p.y, p.z))
    box = np.array([0, 1, 0, 1, 0, 1], np.float32)
    compare(oracle, x, y, z, p.m, p.h, box, shells=1, force_tol=1e-4)
