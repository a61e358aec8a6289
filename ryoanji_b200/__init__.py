"""ryoanji-b200: the single-GPU Barnes-Hut gravity path of Ryoanji/Cornerstone for NVIDIA B200 (sm_100a).

Python host mirror of the C ABI in include/ryoanji_b200.h. Device arrays are torch CUDA tensors (torch is used for
device memory and streams only); every computation runs in the library's own sm_100a kernels. Names follow the
reference (cstone::computeSfcKeys, computeOctree, buildOctreeGpu, ryoanji::TreeBuilder, traverse,
computeGravityEwaldGpu, directSum, ...). Functions raise RyoError on a failed status; the library must be built
(python -m ryoanji_b200.build) and is never replaced by a CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._abi import (BOUNDARY_CUBIC_OPEN, BOUNDARY_FIXED, BOUNDARY_OPEN, BOUNDARY_PERIODIC, RyoError, lib)

__all__ = [
    "Box", "Context", "RyoError", "TreeBuilder", "SolveParams", "SolveResult", "EwaldSettings", "lib",
    "default_context",
    "compute_sfc_keys", "compute_bounding_box", "sequence", "sort_by_key", "compute_octree", "build_octree",
    "compute_fixed_groups", "compute_group_splits", "compute_leaf_source_center", "upsweep_centers",
    "compute_leaf_multipoles", "upsweep_multipoles", "set_mac", "traverse", "read_bh_stats",
    "read_traversal_retries", "bh_max_target_size", "stack_size",
    "compute_gravity_ewald", "ewald_targets_f64", "direct_sum", "direct_targets_f64",
    "solve", "solve_host", "solve_targets", "solve_arrays", "solve_batch", "BatchSystem", "BatchResult", "Engine",
    "kernel_launches", "measure_peaks",
    "BOUNDARY_OPEN", "BOUNDARY_PERIODIC", "BOUNDARY_FIXED", "BOUNDARY_CUBIC_OPEN", "MAX_TREE_LEVEL",
]

MAX_TREE_LEVEL = 21


def _stream(stream=None, ctx: "Context | None" = None) -> C.c_void_p:
    """the caller's stream, else the current stream of the context's device (of the current device without one)"""
    s = stream if stream is not None else torch.cuda.current_stream(ctx.device if ctx is not None else None)
    return C.c_void_p(s.cuda_stream)


def _ptr(t: torch.Tensor | None) -> C.c_void_p | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _check(status: int, ctx: "Context | None" = None) -> None:
    if status != 0:
        msg = lib.ryo_ctx_last_error(ctx.handle if ctx is not None else None)
        raise RyoError(status, (msg or b"").decode(errors="replace"))


def _same_device(ctx: "Context", *tensors) -> None:
    """a context's calls run on the context's device, so its device arrays must live there"""
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda and t.device.index != ctx.device:
            raise ValueError(f"a tensor on {t.device} was passed with a context on cuda:{ctx.device}")


@dataclass
class Box:
    """cstone::Box (cstone/include/cstone/sfc/box.hpp:99-214): limits x0, x1, y0, y1, z0, z1 and boundaries"""

    xmin: float
    xmax: float
    ymin: float
    ymax: float
    zmin: float
    zmax: float
    boundary: tuple = (BOUNDARY_OPEN, BOUNDARY_OPEN, BOUNDARY_OPEN)

    @classmethod
    def cube(cls, lo: float, hi: float, boundary: int = BOUNDARY_OPEN) -> "Box":
        return cls(lo, hi, lo, hi, lo, hi, (boundary,) * 3)

    @property
    def limits(self):
        return [self.xmin, self.xmax, self.ymin, self.ymax, self.zmin, self.zmax]

    @property
    def lengths(self):
        return [self.xmax - self.xmin, self.ymax - self.ymin, self.zmax - self.zmin]

    @property
    def periodic(self) -> bool:
        return all(b == BOUNDARY_PERIODIC for b in self.boundary)

    def f32(self) -> _abi.BoxF32:
        b = _abi.BoxF32()
        for i, v in enumerate(self.limits):
            b.limits[i] = v
        for i, v in enumerate(self.boundary):
            b.boundary[i] = v
        return b

    def f64(self) -> _abi.BoxF64:
        b = _abi.BoxF64()
        for i, v in enumerate(self.limits):
            b.limits[i] = v
        for i, v in enumerate(self.boundary):
            b.boundary[i] = v
        return b


@dataclass
class EwaldSettings:
    """ryoanji::EwaldSettings (ryoanji/src/ryoanji/nbody/ewald.h:23-31)"""

    numReplicaShells: int = 1
    lCut: float = 2.6
    hCut: float = 2.8
    alpha_scale: float = 2.0
    small_R_scale_factor: float = 3.0e-3

    def c(self) -> _abi.EwaldSettings:
        return _abi.EwaldSettings(self.numReplicaShells, self.lCut, self.hCut, self.alpha_scale,
                                  self.small_R_scale_factor)


class Context:
    """Per-device scratch memory, counters and statistics (independent of other contexts)."""

    def __init__(self, device: int | None = None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = device
        h = C.c_void_p()
        _check(lib.ryo_ctx_create(device, C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib.ryo_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


# ---------------------------------------------------------------------------------------------------- cstone layer

def compute_sfc_keys(x, y, z, box: Box, keys=None, stream=None) -> torch.Tensor:
    """cstone::computeSfcKeys: 64-bit Hilbert keys; keys already equal to 2^63 are kept"""
    n = x.numel()
    if keys is None:
        keys = torch.zeros(n, dtype=torch.int64, device=x.device)
    if x.dtype == torch.float32:
        b = box.f32()
        _check(lib.ryo_compute_sfc_keys_f32(_ptr(x), _ptr(y), _ptr(z), _ptr(keys), C.c_size_t(n), C.byref(b),
                                            _stream(stream)))
    elif x.dtype == torch.float64:
        b = box.f64()
        _check(lib.ryo_compute_sfc_keys_f64(_ptr(x), _ptr(y), _ptr(z), _ptr(keys), C.c_size_t(n), C.byref(b),
                                            _stream(stream)))
    else:
        raise TypeError("coordinates must be float32 or float64")
    return keys


def compute_bounding_box(x, y, z, ctx: Context | None = None, stream=None) -> list[float]:
    ctx = ctx or default_context()
    _same_device(ctx, x, y, z)
    out = (C.c_float * 6)()
    _check(lib.ryo_compute_bounding_box_f32(ctx.handle, _ptr(x), _ptr(y), _ptr(z), C.c_size_t(x.numel()), out,
                                            _stream(stream, ctx)), ctx)
    return list(out)


def sequence(n: int, first: int = 0, device=None, stream=None) -> torch.Tensor:
    v = torch.empty(n, dtype=torch.int32, device=device or "cuda")
    _check(lib.ryo_sequence(_ptr(v), C.c_size_t(n), C.c_uint32(first), _stream(stream)))
    return v


def sort_by_key(keys: torch.Tensor, values: torch.Tensor, stream=None) -> None:
    """stable ascending sort of int64/uint64 keys carrying int32 values, in place (cstone::sortByKey)"""
    n = keys.numel()
    kb = torch.empty_like(keys)
    vb = torch.empty_like(values)
    tmp = torch.empty(int(lib.ryo_sort_by_key_temp_bytes(C.c_size_t(n))), dtype=torch.uint8, device=keys.device)
    _check(lib.ryo_sort_by_key(_ptr(keys), _ptr(values), C.c_size_t(n), _ptr(kb), _ptr(vb), _ptr(tmp),
                               C.c_size_t(tmp.numel()), _stream(stream)))


def compute_octree(sorted_keys: torch.Tensor, bucket_size: int, ctx: Context | None = None, stream=None):
    """cstone::computeOctree on the GPU: (leaves[numLeaves + 1] int64, counts[numLeaves] int32)"""
    ctx = ctx or default_context()
    _same_device(ctx, sorted_keys)
    n = sorted_keys.numel()
    num = C.c_int(0)
    st = lib.ryo_compute_octree(ctx.handle, _ptr(sorted_keys), C.c_size_t(n), C.c_uint(bucket_size), None, None, 0,
                                C.byref(num), _stream(stream, ctx))
    if st not in (0, _abi.ERR_CAPACITY):
        _check(st, ctx)
    leaves = torch.empty(num.value + 1, dtype=torch.int64, device=sorted_keys.device)
    counts = torch.empty(num.value, dtype=torch.int32, device=sorted_keys.device)
    _check(lib.ryo_compute_octree(ctx.handle, _ptr(sorted_keys), C.c_size_t(n), C.c_uint(bucket_size), _ptr(leaves),
                                  _ptr(counts), num.value, C.byref(num), _stream(stream, ctx)), ctx)
    return leaves, counts


def build_octree(leaves: torch.Tensor, ctx: Context | None = None, stream=None) -> dict:
    """cstone::buildOctreeGpu: the linked octree of a cornerstone leaf array"""
    ctx = ctx or default_context()
    _same_device(ctx, leaves)
    nl = leaves.numel() - 1
    ni = (nl - 1) // 7
    nn = nl + ni
    dev = leaves.device
    t = dict(
        prefixes=torch.empty(nn, dtype=torch.int64, device=dev),
        childOffsets=torch.empty(nn + 1, dtype=torch.int32, device=dev),
        parents=torch.empty(max(1, (nn - 1) // 8), dtype=torch.int32, device=dev),
        d_levelRange=torch.empty(MAX_TREE_LEVEL + 2, dtype=torch.int32, device=dev),
        internalToLeaf=torch.empty(nn, dtype=torch.int32, device=dev),
        leafToInternal=torch.empty(nn, dtype=torch.int32, device=dev),
    )
    lr = (C.c_int * (MAX_TREE_LEVEL + 2))()
    _check(lib.ryo_build_octree(ctx.handle, _ptr(leaves), nl, _ptr(t["prefixes"]), _ptr(t["childOffsets"]),
                                _ptr(t["parents"]), lr, _ptr(t["d_levelRange"]), _ptr(t["internalToLeaf"]),
                                _ptr(t["leafToInternal"]), _stream(stream, ctx)), ctx)
    t["childOffsets"] = t["childOffsets"][:nn]
    t.update(levelRange=list(lr), numLeafNodes=nl, numInternalNodes=ni, numNodes=nn)
    return t


def compute_fixed_groups(first: int, last: int, group_size: int, device=None, stream=None) -> torch.Tensor:
    """cstone::computeFixedGroups: groups[numGroups + 1]; groupStart = groups[:-1], groupEnd = groups[1:]"""
    ng = (last - first + group_size - 1) // group_size
    g = torch.empty(ng + 1, dtype=torch.int32, device=device or "cuda")
    _check(lib.ryo_compute_fixed_groups(C.c_uint32(first), C.c_uint32(last), C.c_uint(group_size), _ptr(g),
                                        _stream(stream)))
    return g


def compute_group_splits(x, y, z, h, leaves, layout, box: Box, group_size: int = 64, tol_factor: float = 2.0,
                         extent_ratio: float = -1.0, first: int = 0, last: int | None = None,
                         ctx: Context | None = None, stream=None) -> torch.Tensor:
    """cstone::computeGroupSplits: spatial target groups of SFC-sorted bodies (int32 tensor of numGroups + 1
    entries: group starts, then last); leaves/layout are the cornerstone leaf array and body layout"""
    ctx = ctx or default_context()
    _same_device(ctx, x, y, z, h, leaves, layout)
    last = x.numel() if last is None else last
    cap = (last - first) + 2
    groups = torch.empty(cap, dtype=torch.int32, device=x.device)
    num = C.c_uint32(0)
    bx = box.f32()
    _check(lib.ryo_compute_group_splits_f32(ctx.handle, C.c_uint32(first), C.c_uint32(last), _ptr(x), _ptr(y),
                                            _ptr(z), _ptr(h), _ptr(leaves), C.c_int(leaves.numel() - 1),
                                            _ptr(layout), C.byref(bx), C.c_uint(group_size), C.c_float(tol_factor),
                                            C.c_float(extent_ratio), _ptr(groups), C.c_uint32(cap), C.byref(num),
                                            _stream(stream, ctx)), ctx)
    return groups[:num.value + 1]


# ---------------------------------------------------------------------------------------------------- upsweep

def _type_set(x, m) -> str:
    """the reference's type set of a step from its coordinate and mass dtypes: f32, f64 or mixed (double
    coordinates, float masses)"""
    if x.dtype == torch.float32:
        return "f32"
    if x.dtype == torch.float64:
        return "f64" if m is None or m.dtype == torch.float64 else "mixed"
    raise TypeError("coordinates must be float32 or float64")


def compute_leaf_source_center(x, y, z, m, leaf_to_internal, layout, centers, stream=None):
    """cstone::computeLeafSourceCenterGpu; float32 coordinates give float centres, float64 coordinates double
    centres (masses float64 or float32)"""
    nl = leaf_to_internal.numel()
    fn = getattr(lib, "ryo_compute_leaf_source_center_" + _type_set(x, m))
    _check(fn(_ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(leaf_to_internal), nl, _ptr(layout), _ptr(centers),
              _stream(stream)))


def upsweep_centers(num_levels: int, level_range, child_offsets, centers, stream=None):
    lr = (C.c_int * (MAX_TREE_LEVEL + 2))(*level_range)
    fn = lib.ryo_upsweep_centers_f64 if centers.dtype == torch.float64 else lib.ryo_upsweep_centers_f32
    _check(fn(num_levels, lr, _ptr(child_offsets), _ptr(centers), _stream(stream)))


def compute_leaf_multipoles(x, y, z, m, leaf_to_internal, layout, centers, multipoles, stream=None, mdq=False):
    """ryoanji::computeLeafMultipoles: 8 values per node, or 12 with mdq (CartesianMDQpole); the type set follows
    the coordinates and masses (f32, f64, or mixed: double coordinates and centres, float masses and multipoles)"""
    nl = leaf_to_internal.numel()
    fn = getattr(lib, "ryo_compute_leaf_multipoles_" + ("mdq_" if mdq else "") + _type_set(x, m))
    _check(fn(_ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(leaf_to_internal), nl, _ptr(layout), _ptr(centers),
              _ptr(multipoles), _stream(stream)))


def upsweep_multipoles(first_cell: int, last_cell: int, child_offsets, centers, multipoles, stream=None, mdq=False):
    """ryoanji::upsweepMultipoles for the cells [first_cell, last_cell) of one level; double centres with double
    multipoles are the f64 set, double centres with float multipoles the mixed one"""
    kind = "f32" if centers.dtype == torch.float32 else ("f64" if multipoles.dtype == torch.float64 else "mixed")
    fn = getattr(lib, "ryo_upsweep_multipoles_" + ("mdq_" if mdq else "") + kind)
    _check(fn(first_cell, last_cell, _ptr(child_offsets), _ptr(centers), _ptr(multipoles), _stream(stream)))


def set_mac(prefixes, centers, inv_theta: float, box: Box, stream=None):
    if centers.dtype == torch.float64:
        b = box.f64()
        fn = lib.ryo_set_mac_f64
    else:
        b = box.f32()
        fn = lib.ryo_set_mac_f32
    _check(fn(_ptr(prefixes), prefixes.numel(), _ptr(centers), C.c_float(inv_theta), C.byref(b), _stream(stream)))


# ---------------------------------------------------------------------------------------------------- traversal

def bh_max_target_size() -> int:
    return lib.ryo_bh_max_target_size()


def stack_size(num_groups: int) -> int:
    return lib.ryo_stack_size(C.c_uint32(num_groups))


def traverse(groups: torch.Tensor, init_node: int, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, child_offsets,
             internal_to_leaf, layout, source_center, multipoles, G: float, num_shells: int, box_l, p, ax, ay, az,
             ctx: Context | None = None, stack_capacity: int = 0, group_counts: bool = False, first_body: int = 0,
             last_body: int | None = None, stream=None, mdq: bool = False):
    """ryoanji::traverse: accumulates G m phi into p (may be None) and G a into ax, ay, az.

    The instantiation follows the dtypes (traversal_gpu.cu:635-641): float32 everything; float64 everything; or
    float64 coordinates and centres with float32 masses, softenings, multipoles and outputs ("mixed").

    ``groups`` holds numGroups + 1 boundaries (computeFixedGroups layout). Returns the total potential
    0.5 G sum(m phi) and, with group_counts, the per-group (M2P cells, P2P bodies) counts.
    """
    ctx = ctx or default_context()
    _same_device(ctx, groups, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, child_offsets, internal_to_leaf, layout, source_center,
                 multipoles, p, ax, ay, az)
    ng = groups.numel() - 1
    gv = _abi.GroupView(first_body, last_body if last_body is not None else xt.numel(), ng,
                        C.c_void_p(groups.data_ptr()), C.c_void_p(groups.data_ptr() + 4))
    opts = _abi.TraverseOptions()
    opts.multipole = _abi.MULTIPOLE_MDQ if mdq else _abi.MULTIPOLE_QUADRUPOLE
    m2p = p2p = None
    if group_counts:
        m2p = torch.zeros(ng, dtype=torch.int32, device=groups.device)
        p2p = torch.zeros(ng, dtype=torch.int32, device=groups.device)
        opts.groupM2P = C.c_void_p(m2p.data_ptr())
        opts.groupP2P = C.c_void_p(p2p.data_ptr())
    opts.stackCapacity = stack_capacity
    kind = _type_set(xt, mt)
    real = C.c_float if kind == "f32" else C.c_double
    bl = (real * 3)(*(list(box_l) if box_l is not None else [0.0, 0.0, 0.0]))
    pot = C.c_double(0)
    fn = {"f32": lib.ryo_traverse_ex_f32, "f64": lib.ryo_traverse_f64, "mixed": lib.ryo_traverse_mixed}[kind]
    _check(fn(ctx.handle, C.byref(gv), init_node, _ptr(xt), _ptr(yt), _ptr(zt), _ptr(mt), _ptr(ht), _ptr(xs),
              _ptr(ys), _ptr(zs), _ptr(ms), _ptr(hs), _ptr(child_offsets), _ptr(internal_to_leaf), _ptr(layout),
              _ptr(source_center), _ptr(multipoles), real(G), num_shells, bl, _ptr(p), _ptr(ax), _ptr(ay), _ptr(az),
              C.byref(pot), C.byref(opts), _stream(stream, ctx)), ctx)
    if group_counts:
        return pot.value, m2p, p2p
    return pot.value


def read_bh_stats(ctx: Context | None = None) -> list[int]:
    """ryoanji::readBhStats: sumP2P, maxP2P, sumM2P, maxM2P, maxStack of the last traversal"""
    ctx = ctx or default_context()
    out = (C.c_uint64 * 5)()
    _check(lib.ryo_read_bh_stats(ctx.handle, out), ctx)
    return list(out)


def read_traversal_retries(ctx: Context | None = None) -> int:
    ctx = ctx or default_context()
    return int(lib.ryo_read_traversal_retries(ctx.handle))


# ---------------------------------------------------------------------------------------------------- Ewald, direct

def compute_gravity_ewald(root_center, m_root, groups: torch.Tensor, x, y, z, m, box: Box, G: float, ugrav, ax, ay,
                          az, settings: EwaldSettings | None = None, ctx: Context | None = None, stream=None) -> float:
    """ryoanji::computeGravityEwaldGpu; returns the Ewald potential energy 0.5 G sum(m phi_ewald)"""
    ctx = ctx or default_context()
    _same_device(ctx, groups, x, y, z, m, ugrav, ax, ay, az)
    settings = settings or EwaldSettings()
    ng = groups.numel() - 1
    gv = _abi.GroupView(0, x.numel(), ng, C.c_void_p(groups.data_ptr()), C.c_void_p(groups.data_ptr() + 4))
    kind = _type_set(x, m)  # f32, f64 (double everything) or mixed (double coordinates, float masses and outputs)
    real = C.c_float if kind == "f32" else C.c_double
    rc = (real * 3)(*[float(v) for v in root_center])
    mr = ((C.c_double if kind == "f64" else C.c_float) * 8)(*[float(v) for v in m_root])
    b = box.f32() if kind == "f32" else box.f64()
    tot = C.c_double(0)
    s = settings.c()
    fn = getattr(lib, "ryo_compute_gravity_ewald_" + kind)
    _check(fn(ctx.handle, rc, mr, C.byref(gv), _ptr(x), _ptr(y), _ptr(z), _ptr(m), C.byref(b), C.c_float(G),
              _ptr(ugrav), _ptr(ax), _ptr(ay), _ptr(az), C.byref(tot), C.byref(s), _stream(stream, ctx)), ctx)
    return tot.value


def direct_sum(first: int, last: int, num_bodies: int, box_l, num_shells: int, x, y, z, m, h, p, ax, ay, az,
               stream=None):
    """ryoanji::directSum: adds m phi to p and a to ax, ay, az for targets [first, last) (no G)"""
    if x.dtype == torch.float32:
        bl = (C.c_float * 3)(*box_l)
        fn = lib.ryo_direct_sum_f32
    else:
        bl = (C.c_double * 3)(*box_l)
        fn = lib.ryo_direct_sum_f64
    _check(fn(C.c_size_t(first), C.c_size_t(last), C.c_size_t(num_bodies), bl, num_shells, _ptr(x), _ptr(y), _ptr(z),
              _ptr(m), _ptr(h), _ptr(p), _ptr(ax), _ptr(ay), _ptr(az), _stream(stream)))


def direct_targets_f64(targets: torch.Tensor, x, y, z, m, h, G: float = 1.0, box_l=(0.0, 0.0, 0.0),
                       num_shells: int = 0, stream=None):
    """double-precision direct sum for chosen targets of float data: (pot, ax, ay, az) float64 tensors"""
    nt = targets.numel()
    out = [torch.empty(nt, dtype=torch.float64, device=x.device) for _ in range(4)]
    bl = (C.c_double * 3)(*box_l)
    _check(lib.ryo_direct_targets_f64(_ptr(targets), C.c_size_t(nt), _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(h),
                                      C.c_size_t(x.numel()), C.c_double(G), bl, num_shells, *[_ptr(o) for o in out],
                                      _stream(stream)))
    return out


def ewald_targets_f64(targets: torch.Tensor, x, y, z, m, h, L: float, G: float = 1.0,
                      ewald: "EwaldSettings | None" = None, ctx: Context | None = None, stream=None):
    """FP64 periodic sum for chosen targets of a cubic box [x0, x0 + L)^3: direct sum over the replica shells plus
    the particle-level Ewald correction; (pot = G m phi, ax, ay, az) float64 tensors"""
    ctx = ctx or default_context()
    _same_device(ctx, targets, x, y, z, m, h)
    e = (ewald or EwaldSettings()).c()
    out = direct_targets_f64(targets, x, y, z, m, h, G=G, box_l=(L, L, L), num_shells=e.numReplicaShells,
                             stream=stream)
    _check(lib.ryo_ewald_targets_f64(ctx.handle, _ptr(targets), C.c_size_t(targets.numel()), _ptr(x), _ptr(y),
                                     _ptr(z), _ptr(m), C.c_size_t(x.numel()), C.c_double(L), C.byref(e),
                                     C.c_double(G), *[_ptr(o) for o in out], _stream(stream, ctx)), ctx)
    return out


# ---------------------------------------------------------------------------------------------------- TreeBuilder

class TreeBuilder:
    """ryoanji::TreeBuilder<uint64_t> (ryoanji/src/ryoanji/interface/treebuilder.cuh:34-125)"""

    def __init__(self, ncrit: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        _check(lib.ryo_treebuilder_create(self.ctx.handle, ncrit, C.byref(h)), self.ctx)
        self.handle = h
        self._view = None

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib.ryo_treebuilder_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def update(self, x, y, z, box: Box, stream=None) -> int:
        """sorts x, y, z in place into SFC order and builds the tree; returns the number of nodes"""
        _same_device(self.ctx, x, y, z)
        nn = C.c_int(0)
        if x.dtype == torch.float32:
            b = box.f32()
            fn = lib.ryo_treebuilder_update_f32
        else:
            b = box.f64()
            fn = lib.ryo_treebuilder_update_f64
        _check(fn(self.handle, _ptr(x), _ptr(y), _ptr(z), C.c_size_t(x.numel()), C.byref(b), C.byref(nn),
                  _stream(stream, self.ctx)), self.ctx)
        v = _abi.TreeView()
        _check(lib.ryo_treebuilder_view(self.handle, C.byref(v)))
        self._view = v
        self._n = x.numel()
        self._device = x.device
        return nn.value

    def _wrap(self, ptr, count, dtype):
        return _abi.wrap_device(ptr, count, dtype, self._device)

    @property
    def numLeafNodes(self) -> int:
        return self._view.numLeafNodes

    @property
    def numNodes(self) -> int:
        return self._view.numNodes

    @property
    def maxTreeLevel(self) -> int:
        return self._view.maxTreeLevel

    @property
    def levelRange(self) -> list[int]:
        return list(self._view.levelRange)

    def layout(self) -> torch.Tensor:
        return self._wrap(self._view.layout, self.numLeafNodes + 1, torch.int32)

    def nodeKeys(self) -> torch.Tensor:
        return self._wrap(self._view.nodeKeys, self.numNodes, torch.int64)

    def childOffsets(self) -> torch.Tensor:
        return self._wrap(self._view.childOffsets, self.numNodes, torch.int32)

    def leafToInternal(self) -> torch.Tensor:
        return self._wrap(self._view.leafToInternal, self.numLeafNodes, torch.int32)

    def internalToLeaf(self) -> torch.Tensor:
        return self._wrap(self._view.internalToLeaf, self.numNodes, torch.int32)

    def parents(self) -> torch.Tensor:
        return self._wrap(self._view.parents, max(1, (self.numNodes - 1) // 8), torch.int32)

    def leaves(self) -> torch.Tensor:
        return self._wrap(self._view.leaves, self.numLeafNodes + 1, torch.int64)

    def order(self) -> torch.Tensor:
        return self._wrap(self._view.order, self._n, torch.int32)

    def sortedKeys(self) -> torch.Tensor:
        return self._wrap(self._view.sortedKeys, self._n, torch.int64)


# ---------------------------------------------------------------------------------------------------- fused solve

@dataclass
class SolveParams:
    bucket_size: int = 64
    group_size: int = 64
    theta: float = 0.5
    G: float = 1.0
    box: Box | None = None
    num_shells: int = 1
    ewald: EwaldSettings | None = None
    stack_capacity: int = 0
    timing: bool = False
    group_tolerance: float = 0.0  # > 0: spatial target groups with this tolFactor (the reference's production uses 2)
    group_extent_ratio: float = -1.0  # < 0: the reference default
    multipole: str = "quadrupole"  # or "mdq": monopole + dipole + quadrupole (CartesianMDQpole), for signed masses

    def c(self) -> _abi.SolveParams:
        p = _abi.SolveParams()
        lib.ryo_solve_params_default(C.byref(p))
        p.bucketSize = self.bucket_size
        p.groupSize = self.group_size
        p.theta = self.theta
        p.G = self.G
        if self.box is not None:
            p.useBox = 1
            p.box = self.box.f32()
        p.numShells = self.num_shells
        if self.ewald is not None:
            p.ewald = self.ewald.c()
        p.stackCapacity = self.stack_capacity
        p.timing = int(self.timing)
        p.groupTolerance = self.group_tolerance
        p.groupExtentRatio = self.group_extent_ratio
        p.multipole = {"quadrupole": _abi.MULTIPOLE_QUADRUPOLE, "mdq": _abi.MULTIPOLE_MDQ}[self.multipole]
        return p


@dataclass
class SolveResult:
    num_leaves: int
    num_nodes: int
    num_groups: int
    sum_p2p: int
    max_p2p: int
    sum_m2p: int
    max_m2p: int
    max_stack: int
    retries: int
    potential_energy: float
    box: list
    ms: dict


def solve(x, y, z, m, h, p, ax, ay, az, params: SolveParams | None = None, v=None, order=None,
          ctx: Context | None = None, stream=None) -> SolveResult:
    """The fused single-system solve. x, y, z, m, h (and v = (vx, vy, vz) if given) are sorted in place into SFC
    order; p, ax, ay, az receive G m phi and G a in that order; order (int32, optional) the original indices."""
    ctx = ctx or default_context()
    _same_device(ctx, x, y, z, m, h, p, ax, ay, az, order, *(v or ()))
    params = params or SolveParams()
    pc = params.c()
    st = _abi.SolveStats()
    vx, vy, vz = v if v is not None else (None, None, None)
    _check(lib.ryo_solve_f32(ctx.handle, C.byref(pc), _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(h), _ptr(vx), _ptr(vy),
                             _ptr(vz), C.c_size_t(x.numel()), _ptr(p), _ptr(ax), _ptr(ay), _ptr(az), _ptr(order),
                             C.byref(st), _stream(stream, ctx)), ctx)
    _solve_n[id(ctx)] = x.numel()
    ms = dict(zip(("sort", "tree", "upsweep", "traverse", "ewald", "total"), list(st.ms)))
    return SolveResult(st.numLeaves, st.numNodes, st.numGroups, st.sumP2P, st.maxP2P, st.sumM2P, st.maxM2P,
                       st.maxStack, st.retries, st.potentialEnergy, list(st.box), ms)


def solve_host(x, y, z, m, h, p, ax, ay, az, params: SolveParams | None = None, sorted_xyz=None, order=None,
               ctx: Context | None = None, stream=None) -> SolveResult:
    """The fused solve from and to host memory (ryo_solve_host_f32): x, y, z, m, h are contiguous host float32
    arrays (CPU tensors, pinned for the fastest copies), left unchanged; p, ax, ay, az (host float32) receive G m phi
    and G a in SFC order, sorted_xyz (three host arrays, optional) the positions in that order and order (host
    int32, optional) the original index of each sorted body. Host copies overlap the solve; pinned p, ax, ay, az
    of an open system receive the traversal's results directly. Returns when every output is in host memory."""
    ctx = ctx or default_context()
    params = params or SolveParams()
    for a in (x, y, z, m, h, p, ax, ay, az) + tuple(sorted_xyz or ()) + ((order,) if order is not None else ()):
        if not (isinstance(a, torch.Tensor) and a.device.type == "cpu" and a.is_contiguous() and
                a.numel() == x.numel() and a.element_size() == 4):
            raise ValueError("solve_host: every array must be a contiguous 4-byte CPU tensor of n elements")
    pc = params.c()
    st = _abi.SolveStats()
    xs, ys, zs = sorted_xyz if sorted_xyz is not None else (None, None, None)
    hp = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731  (host pointers, checked above)
    _check(lib.ryo_solve_host_f32(ctx.handle, C.byref(pc), hp(x), hp(y), hp(z), hp(m), hp(h), C.c_size_t(x.numel()),
                                  hp(xs), hp(ys), hp(zs), hp(p), hp(ax), hp(ay), hp(az), hp(order), C.byref(st),
                                  _stream(stream, ctx)), ctx)
    _solve_n[id(ctx)] = x.numel()
    ms = dict(zip(("sort", "tree", "upsweep", "traverse", "ewald", "total"), list(st.ms)))
    return SolveResult(st.numLeaves, st.numNodes, st.numGroups, st.sumP2P, st.maxP2P, st.sumM2P, st.maxM2P,
                       st.maxStack, st.retries, st.potentialEnergy, list(st.box), ms)


@dataclass
class BatchSystem:
    """one system of a batched solve: @p num_bodies consecutive bodies; box None means the enclosing cube"""
    num_bodies: int
    box: Box | None = None
    num_shells: int = 1


@dataclass
class BatchResult:
    stats: SolveResult
    energies: list
    boxes: list


MAX_BATCH_SYSTEMS = 4096


def solve_batch(systems, x, y, z, m, h, p, ax, ay, az, params: SolveParams | None = None, v=None, order=None,
                ctx: Context | None = None, stream=None) -> BatchResult:
    """Solve many independent systems in one launch per phase. The arrays hold the systems' bodies concatenated in
    the order of @p systems (a list of BatchSystem); each system is sorted in place within its own range."""
    ctx = ctx or default_context()
    _same_device(ctx, x, y, z, m, h, p, ax, ay, az, order, *(v or ()))
    params = params or SolveParams()
    pc = params.c()
    ns = len(systems)
    arr = (_abi.System * max(ns, 1))()
    first = 0
    for i, sy in enumerate(systems):
        arr[i].firstBody = first
        arr[i].numBodies = int(sy.num_bodies)
        arr[i].useBox = 1 if sy.box is not None else 0
        if sy.box is not None:
            arr[i].box = sy.box.f32()
        arr[i].numShells = int(sy.num_shells)
        first += int(sy.num_bodies)
    energies = (C.c_double * max(ns, 1))()
    boxes = (C.c_float * (6 * max(ns, 1)))()
    st = _abi.SolveStats()
    vx, vy, vz = v if v is not None else (None, None, None)
    _check(lib.ryo_solve_batch_f32(ctx.handle, C.byref(pc), arr, ns, _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(h),
                                   _ptr(vx), _ptr(vy), _ptr(vz), C.c_size_t(x.numel()), _ptr(p), _ptr(ax), _ptr(ay),
                                   _ptr(az), _ptr(order), energies, boxes, C.byref(st), _stream(stream, ctx)), ctx)
    ms = dict(zip(("sort", "tree", "upsweep", "traverse", "ewald", "total"), list(st.ms)))
    res = SolveResult(st.numLeaves, st.numNodes, st.numGroups, st.sumP2P, st.maxP2P, st.sumM2P, st.maxM2P,
                      st.maxStack, st.retries, st.potentialEnergy, [], ms)
    return BatchResult(res, list(energies)[:ns], [list(boxes[6 * i:6 * i + 6]) for i in range(ns)])


class Engine:
    """The served stream (ryo_engine_*): requests of a particle set and K leapfrog steps, admitted under an HBM
    budget and advanced together, one batched solve per step. Host inputs are kept referenced until admission and
    output buffers until retirement."""

    def __init__(self, params: SolveParams | None = None, hbm_budget_bytes: float = 120e9,
                 bytes_per_body: float = 256.0, max_systems: int = MAX_BATCH_SYSTEMS, ctx: Context | None = None,
                 reserve_bodies: int = 0, max_step_bodies: int | None = None):
        """max_step_bodies: bodies one step advances at most (None: the library default, 7 x 2^20; 0: every resident
        request every step); the requests with the least remaining work go first"""
        self.ctx = ctx or default_context()
        ep = _abi.EngineParams()
        lib.ryo_engine_params_default(C.byref(ep))
        ep.solve = (params or SolveParams()).c()
        ep.hbmBudgetBytes = hbm_budget_bytes
        ep.bytesPerBody = bytes_per_body
        ep.maxSystems = max_systems
        ep.reserveBodies = reserve_bodies
        if max_step_bodies is not None:
            ep.maxStepBodies = max_step_bodies
        h = C.c_void_p()
        _check(lib.ryo_engine_create(self.ctx.handle, C.byref(ep), C.byref(h)), self.ctx)
        self.handle = h
        self._keep = {}
        self._outputs = {}

    def _err(self, st):
        if st != 0:
            raise RyoError(st, (lib.ryo_engine_last_error(self.handle) or b"").decode(errors="replace"))

    def submit(self, tag: int, x, y, z, m, h, vx=None, vy=None, vz=None, box: Box | None = None, num_shells: int = 1,
               steps: int = 1, dt: float = 1e-3, want_output: bool = False, out=None):
        """queue one request; arrays are host float32 (numpy or CPU tensors, pinned memory copies fastest).
        With want_output, the final state goes to @p out (a contiguous host float32 array or tensor of 10 x n,
        pinned for the fastest copy) or to a new numpy array."""
        def host(a):
            if a is None:
                return None
            if isinstance(a, torch.Tensor):
                assert a.device.type == "cpu" and a.dtype == torch.float32 and a.is_contiguous()
                return a
            return np.ascontiguousarray(a, dtype=np.float32)

        arrs = [host(a) for a in (x, y, z, m, h, vx, vy, vz)]
        ptr = lambda a: None if a is None else (a.data_ptr() if isinstance(a, torch.Tensor)  # noqa: E731
                                                  else a.ctypes.data)
        r = _abi.EngineRequest()
        r.tag = tag
        r.numBodies = len(arrs[0])
        for k, a in zip(("x", "y", "z", "m", "h", "vx", "vy", "vz"), arrs):
            setattr(r, k, ptr(a))
        r.useBox = 1 if box is not None else 0
        if box is not None:
            r.box = box.f32()
        r.numShells = num_shells
        r.numSteps = steps
        r.dt = dt
        if not want_output:
            out = None
        elif out is None:
            out = np.empty((10, r.numBodies), np.float32)
        else:
            ok = (out.dtype in (np.float32, torch.float32) and tuple(out.shape) == (10, r.numBodies) and
                  (out.is_contiguous() and out.device.type == "cpu" if isinstance(out, torch.Tensor)
                   else out.flags.c_contiguous))
            if not ok:
                raise ValueError("out must be a contiguous host float32 array of shape (10, n)")
        r.out = None if out is None else ptr(out)
        self._err(lib.ryo_engine_submit(self.handle, C.byref(r)))
        self._keep[tag] = arrs
        if out is not None:
            self._outputs[tag] = out

    def step(self, stream=None) -> dict:
        info = _abi.EngineStepInfo()
        self._err(lib.ryo_engine_step(self.handle, C.byref(info), _stream(stream, self.ctx)))
        d = {k: getattr(info, k) for k in ("admitted", "retired", "resident", "queued", "solved", "retries",
                                           "residentBodies", "sumP2P", "maxP2P", "sumM2P", "maxM2P")}
        d["ms"] = list(info.ms)
        d["host_ms"] = list(info.hostMs)
        return d

    def poll(self) -> list:
        """results of retired requests: dicts with tag, bodies, steps, energies and (if requested) the final state
        (x, y, z, vx, vy, vz, ax, ay, az, p as rows of a 10 x n array, submission order)"""
        out = []
        buf = (_abi.EngineResult * 64)()
        while True:
            cnt = C.c_int(0)
            self._err(lib.ryo_engine_poll(self.handle, buf, 64, C.byref(cnt)))
            for i in range(cnt.value):
                r = buf[i]
                self._keep.pop(r.tag, None)
                out.append(dict(tag=r.tag, bodies=r.numBodies, steps=r.stepsDone, kinetic=r.kineticEnergy,
                                potential=r.potentialEnergy, initial=r.initialEnergy,
                                state=self._outputs.pop(r.tag, None)))
            if cnt.value < 64:
                return out

    def status(self) -> dict:
        q, r, b = C.c_int(0), C.c_int(0), C.c_double(0)
        self._err(lib.ryo_engine_status(self.handle, C.byref(q), C.byref(r), C.byref(b)))
        return dict(queued=q.value, resident=r.value, bytes_in_use=b.value)

    def close(self):
        if getattr(self, "handle", None):
            lib.ryo_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_targets(xt, yt, zt, mt=None, ht=None, ctx: Context | None = None, stream=None):
    """field of the last solve() on @p ctx at separate targets (MultipoleHolder::compute with distinct targets):
    (p = G m phi, ax, ay, az) in the targets' order, and the interaction statistics"""
    ctx = ctx or default_context()
    _same_device(ctx, xt, yt, zt, mt, ht)
    n = xt.numel()
    p, ax, ay, az = (torch.empty(n, device=xt.device) for _ in range(4))
    st = _abi.SolveStats()
    _check(lib.ryo_solve_targets_f32(ctx.handle, _ptr(xt), _ptr(yt), _ptr(zt), _ptr(mt), _ptr(ht), C.c_size_t(n),
                                     _ptr(p), _ptr(ax), _ptr(ay), _ptr(az), C.byref(st), _stream(stream, ctx)), ctx)
    res = SolveResult(0, st.numNodes, st.numGroups, st.sumP2P, st.maxP2P, st.sumM2P, st.maxM2P, st.maxStack,
                      st.retries, st.potentialEnergy, list(st.box), {})
    return (p, ax, ay, az), res


_solve_n: dict = {}


def _last_n(ctx) -> int:
    return _solve_n.get(id(ctx), 0)


def kernel_launches() -> int:
    """kernels launched by the library in this process"""
    return int(lib.ryo_kernel_launches())


def measure_peaks(ctx: Context | None = None, stream=None) -> dict:
    """FP32 FMA peak (scalar and packed f32x2) in TFLOP/s and streaming-copy GB/s, measured now"""
    ctx = ctx or default_context()
    out = (C.c_double * 3)()
    _check(lib.ryo_measure_peaks(ctx.handle, out, _stream(stream, ctx)), ctx)
    return dict(fp32_tflops=out[0], fp32x2_tflops=out[1], copy_gbs=out[2])


def solve_arrays(ctx: Context | None = None, device=None) -> dict:
    """torch views of the tree of the last solve on @p ctx (valid until the next solve on it)"""
    ctx = ctx or default_context()
    a = _abi.SolveArrays()
    _check(lib.ryo_solve_arrays_get(ctx.handle, C.byref(a)), ctx)
    dev = device or torch.device("cuda", ctx.device)
    nl, nn, ng = a.numLeaves, a.numNodes, a.numGroups
    w = lambda ptr, cnt, dt: _abi.wrap_device(ptr, cnt, dt, dev)  # noqa: E731
    nd = w(a.nodeData, 16 * nn, torch.float32).view(nn, 16)
    return dict(numLeafNodes=nl, numNodes=nn, numGroups=ng, leaves=w(a.leaves, nl + 1, torch.int64),
                layout=w(a.layout, nl + 1, torch.int32), prefixes=w(a.prefixes, nn, torch.int64),
                childOffsets=w(a.childOffsets, nn, torch.int32), internalToLeaf=w(a.internalToLeaf, nn, torch.int32),
                leafToInternal=w(a.leafToInternal, nn, torch.int32),
                parents=w(a.parents, max(1, (nn - 1) // 8), torch.int32), centers=nd[:, 0:4],
                multipoles=nd[:, 4:12], links=nd[:, 12:16].view(torch.int32), groups=w(a.groups, ng + 1, torch.int32),
                groupM2P=w(a.groupM2P, ng, torch.int32), groupP2P=w(a.groupP2P, ng, torch.int32),
                sortedKeys=w(a.sortedKeys, 0 if not a.sortedKeys else _last_n(ctx), torch.int64),
                levelRange=list(a.levelRange), rootCenter=list(a.rootCenter), rootMultipole=list(a.rootMultipole),
                dipoles=w(a.dipoles, 4 * nn, torch.float32).view(nn, 4) if a.dipoles else None)
