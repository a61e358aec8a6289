"""ctypes declarations of the C ABI (include/ryoanji_b200.h) and the library loader.

The shared library is built in-tree by ``python -m ryoanji_b200.build``. If it is missing the import fails with an
explicit error: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libryoanji_b200.so")

BOUNDARY_OPEN, BOUNDARY_PERIODIC, BOUNDARY_FIXED, BOUNDARY_CUBIC_OPEN = 0, 1, 2, 3
OK, ERR_CUDA, ERR_BAD_ARG, ERR_OOM, ERR_STACK_OVERFLOW, ERR_TIMEOUT, ERR_CAPACITY, ERR_NOT_CUBIC, ERR_NO_DEVICE, \
    ERR_INTERNAL = range(10)


class RyoError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        name = lib.ryo_status_string(status).decode() if lib is not None else str(status)
        super().__init__(f"{name}: {message}" if message else name)


class BoxF32(C.Structure):
    _fields_ = [("limits", C.c_float * 6), ("boundary", C.c_int * 3)]


class BoxF64(C.Structure):
    _fields_ = [("limits", C.c_double * 6), ("boundary", C.c_int * 3)]


class GroupView(C.Structure):
    _fields_ = [("firstBody", C.c_uint32), ("lastBody", C.c_uint32), ("numGroups", C.c_uint32),
                ("groupStart", C.c_void_p), ("groupEnd", C.c_void_p)]


class EwaldSettings(C.Structure):
    _fields_ = [("numReplicaShells", C.c_int), ("lCut", C.c_double), ("hCut", C.c_double),
                ("alpha_scale", C.c_double), ("small_R_scale_factor", C.c_double)]


class TraverseOptions(C.Structure):
    _fields_ = [("groupM2P", C.c_void_p), ("groupP2P", C.c_void_p), ("stackCapacity", C.c_int), ("multipole", C.c_int)]


class TreeView(C.Structure):
    _fields_ = [("numLeafNodes", C.c_int), ("numInternalNodes", C.c_int), ("numNodes", C.c_int),
                ("maxTreeLevel", C.c_uint), ("layout", C.c_void_p), ("nodeKeys", C.c_void_p),
                ("childOffsets", C.c_void_p), ("leafToInternal", C.c_void_p), ("internalToLeaf", C.c_void_p),
                ("parents", C.c_void_p), ("leaves", C.c_void_p), ("order", C.c_void_p), ("sortedKeys", C.c_void_p),
                ("levelRange", C.c_int * 23)]


class SolveParams(C.Structure):
    _fields_ = [("bucketSize", C.c_uint), ("groupSize", C.c_uint), ("theta", C.c_float), ("G", C.c_float),
                ("useBox", C.c_int), ("box", BoxF32), ("numShells", C.c_int), ("ewald", EwaldSettings),
                ("stackCapacity", C.c_int), ("timing", C.c_int), ("groupTolerance", C.c_float),
                ("groupExtentRatio", C.c_float), ("multipole", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("numLeaves", C.c_int), ("numNodes", C.c_int), ("numGroups", C.c_int), ("sumP2P", C.c_uint64),
                ("maxP2P", C.c_uint64), ("sumM2P", C.c_uint64), ("maxM2P", C.c_uint64), ("maxStack", C.c_uint64),
                ("retries", C.c_uint64), ("potentialEnergy", C.c_double), ("box", C.c_float * 6),
                ("ms", C.c_float * 6)]


class SolveArrays(C.Structure):
    _fields_ = [("numLeaves", C.c_int), ("numNodes", C.c_int), ("numGroups", C.c_int), ("sortedKeys", C.c_void_p),
                ("order", C.c_void_p), ("leaves", C.c_void_p), ("layout", C.c_void_p), ("prefixes", C.c_void_p),
                ("childOffsets", C.c_void_p), ("internalToLeaf", C.c_void_p), ("leafToInternal", C.c_void_p),
                ("parents", C.c_void_p), ("nodeData", C.c_void_p), ("groups", C.c_void_p),
                ("groupM2P", C.c_void_p), ("groupP2P", C.c_void_p), ("levelRange", C.c_int * 23),
                ("rootCenter", C.c_double * 3), ("rootMultipole", C.c_double * 8), ("dipoles", C.c_void_p)]


class System(C.Structure):
    _fields_ = [("firstBody", C.c_uint64), ("numBodies", C.c_uint32), ("useBox", C.c_int), ("box", BoxF32),
                ("numShells", C.c_int)]


class EngineParams(C.Structure):
    _fields_ = [("solve", SolveParams), ("hbmBudgetBytes", C.c_double), ("bytesPerBody", C.c_double),
                ("maxSystems", C.c_int), ("reserveBodies", C.c_uint64), ("maxStepBodies", C.c_uint64)]


class EngineRequest(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("numBodies", C.c_uint32)] + [(k, C.c_void_p) for k in
                                                                     ("x", "y", "z", "m", "h", "vx", "vy", "vz")] + \
               [("useBox", C.c_int), ("box", BoxF32), ("numShells", C.c_int), ("numSteps", C.c_int),
                ("dt", C.c_float), ("out", C.c_void_p)]


class EngineStepInfo(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("admitted", "retired", "resident", "queued", "solved", "retries")] + \
               [("residentBodies", C.c_uint64), ("ms", C.c_float * 6)] + \
               [(k, C.c_uint64) for k in ("sumP2P", "maxP2P", "sumM2P", "maxM2P")] + [("hostMs", C.c_float * 4)]


class EngineResult(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("numBodies", C.c_uint32), ("stepsDone", C.c_int),
                ("kineticEnergy", C.c_double), ("potentialEnergy", C.c_double), ("initialEnergy", C.c_double)]


MULTIPOLE_QUADRUPOLE, MULTIPOLE_MDQ = 0, 1

_p = C.c_void_p
_sz = C.c_size_t
_i = C.c_int
_u = C.c_uint
_u32 = C.c_uint32
_f = C.c_float
_d = C.c_double

# name -> (restype, argtypes); every symbol declared in include/ryoanji_b200.h
class LetCounts(C.Structure):
    _fields_ = [("numNodes", C.c_uint32), ("numLeaves", C.c_uint32), ("numBodies", C.c_uint32), ("pad", C.c_uint32),
                ("words", C.c_uint64)]


SIGNATURES = {
    "ryo_status_string": (C.c_char_p, [_i]),
    "ryo_version": (C.c_char_p, []),
    "ryo_ctx_create": (_i, [_i, C.POINTER(_p)]),
    "ryo_ctx_destroy": (None, [_p]),
    "ryo_ctx_last_error": (C.c_char_p, [_p]),
    "ryo_compute_sfc_keys_f32": (_i, [_p, _p, _p, _p, _sz, C.POINTER(BoxF32), _p]),
    "ryo_compute_sfc_keys_f64": (_i, [_p, _p, _p, _p, _sz, C.POINTER(BoxF64), _p]),
    "ryo_compute_bounding_box_f32": (_i, [_p, _p, _p, _p, _sz, C.POINTER(_f), _p]),
    "ryo_sequence": (_i, [_p, _sz, _u32, _p]),
    "ryo_sort_by_key_temp_bytes": (_sz, [_sz]),
    "ryo_sort_by_key": (_i, [_p, _p, _sz, _p, _p, _p, _sz, _p]),
    "ryo_sort_by_key_static": (_i, [_p, _p, _sz, _p, _p, _p]),
    "ryo_sort_wait_timeout_selftest": (_i, [_p]),
    "ryo_compute_octree": (_i, [_p, _p, _sz, _u, _p, _p, _i, C.POINTER(_i), _p]),
    "ryo_build_octree": (_i, [_p, _p, _i, _p, _p, _p, C.POINTER(_i), _p, _p, _p, _p]),
    "ryo_compute_fixed_groups": (_i, [_u32, _u32, _u, _p, _p]),
    "ryo_compute_leaf_source_center_f32": (_i, [_p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "ryo_upsweep_centers_f32": (_i, [_i, C.POINTER(_i), _p, _p, _p]),
    "ryo_compute_leaf_multipoles_f32": (_i, [_p, _p, _p, _p, _p, _i, _p, _p, _p, _p]),
    "ryo_upsweep_multipoles_f32": (_i, [_i, _i, _p, _p, _p, _p]),
    "ryo_compute_leaf_multipoles_mdq_f32": (_i, [_p] * 5 + [_i] + [_p] * 4),
    "ryo_upsweep_multipoles_mdq_f32": (_i, [_i, _i] + [_p] * 4),
    "ryo_set_mac_f32": (_i, [_p, _i, _p, _f, C.POINTER(BoxF32), _p]),
    "ryo_compute_leaf_source_center_f64": (_i, [_p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "ryo_compute_leaf_source_center_mixed": (_i, [_p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "ryo_upsweep_centers_f64": (_i, [_i, C.POINTER(_i), _p, _p, _p]),
    "ryo_compute_leaf_multipoles_f64": (_i, [_p] * 5 + [_i] + [_p] * 4),
    "ryo_compute_leaf_multipoles_mixed": (_i, [_p] * 5 + [_i] + [_p] * 4),
    "ryo_compute_leaf_multipoles_mdq_f64": (_i, [_p] * 5 + [_i] + [_p] * 4),
    "ryo_compute_leaf_multipoles_mdq_mixed": (_i, [_p] * 5 + [_i] + [_p] * 4),
    "ryo_upsweep_multipoles_f64": (_i, [_i, _i] + [_p] * 4),
    "ryo_upsweep_multipoles_mixed": (_i, [_i, _i] + [_p] * 4),
    "ryo_upsweep_multipoles_mdq_f64": (_i, [_i, _i] + [_p] * 4),
    "ryo_upsweep_multipoles_mdq_mixed": (_i, [_i, _i] + [_p] * 4),
    "ryo_set_mac_f64": (_i, [_p, _i, _p, _f, C.POINTER(BoxF64), _p]),
    "ryo_bh_max_target_size": (_i, []),
    "ryo_stack_size": (_u32, [_u32]),
    "ryo_traverse_f32": (_i, [_p, C.POINTER(GroupView), _i] + [_p] * 15 + [_f, _i, C.POINTER(_f), _p, _p, _p, _p,
                                                                            C.POINTER(_d), _p]),
    "ryo_traverse_ex_f32": (_i, [_p, C.POINTER(GroupView), _i] + [_p] * 15 + [_f, _i, C.POINTER(_f), _p, _p, _p, _p,
                                                                               C.POINTER(_d),
                                                                               C.POINTER(TraverseOptions), _p]),
    "ryo_traverse_f64": (_i, [_p, C.POINTER(GroupView), _i] + [_p] * 15 + [_d, _i, C.POINTER(_d), _p, _p, _p, _p,
                                                                           C.POINTER(_d), C.POINTER(TraverseOptions),
                                                                           _p]),
    "ryo_traverse_mixed": (_i, [_p, C.POINTER(GroupView), _i] + [_p] * 15 + [_d, _i, C.POINTER(_d), _p, _p, _p, _p,
                                                                             C.POINTER(_d), C.POINTER(TraverseOptions),
                                                                             _p]),
    "ryo_let_export_f32": (_i, [_p, C.POINTER(_f), _p, C.c_size_t, C.POINTER(LetCounts), _p]),
    "ryo_read_bh_stats": (_i, [_p, C.POINTER(C.c_uint64)]),
    "ryo_read_traversal_retries": (C.c_uint64, [_p]),
    "ryo_compute_gravity_ewald_f32": (_i, [_p, C.POINTER(_f), C.POINTER(_f), C.POINTER(GroupView), _p, _p, _p, _p,
                                           C.POINTER(BoxF32), _f, _p, _p, _p, _p, C.POINTER(_d),
                                           C.POINTER(EwaldSettings), _p]),
    "ryo_compute_gravity_ewald_f64": (_i, [_p, C.POINTER(_d), C.POINTER(_d), C.POINTER(GroupView), _p, _p, _p, _p,
                                           C.POINTER(BoxF64), _f, _p, _p, _p, _p, C.POINTER(_d),
                                           C.POINTER(EwaldSettings), _p]),
    "ryo_compute_gravity_ewald_mixed": (_i, [_p, C.POINTER(_d), C.POINTER(_f), C.POINTER(GroupView), _p, _p, _p, _p,
                                             C.POINTER(BoxF64), _f, _p, _p, _p, _p, C.POINTER(_d),
                                             C.POINTER(EwaldSettings), _p]),
    "ryo_direct_sum_f32": (_i, [_sz, _sz, _sz, C.POINTER(_f), _i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "ryo_direct_sum_f64": (_i, [_sz, _sz, _sz, C.POINTER(_d), _i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "ryo_direct_targets_f64": (_i, [_p, _sz, _p, _p, _p, _p, _p, _sz, _d, C.POINTER(_d), _i, _p, _p, _p, _p, _p]),
    "ryo_treebuilder_create": (_i, [_p, _u, C.POINTER(_p)]),
    "ryo_treebuilder_destroy": (None, [_p]),
    "ryo_treebuilder_update_f32": (_i, [_p, _p, _p, _p, _sz, C.POINTER(BoxF32), C.POINTER(_i), _p]),
    "ryo_treebuilder_update_f64": (_i, [_p, _p, _p, _p, _sz, C.POINTER(BoxF64), C.POINTER(_i), _p]),
    "ryo_treebuilder_view": (_i, [_p, C.POINTER(TreeView)]),
    "ryo_solve_params_default": (None, [C.POINTER(SolveParams)]),
    "ryo_solve_f32": (_i, [_p, C.POINTER(SolveParams)] + [_p] * 8 + [_sz] + [_p] * 5 + [C.POINTER(SolveStats), _p]),
    "ryo_solve_host_f32": (_i, [_p, C.POINTER(SolveParams)] + [_p] * 5 + [_sz] + [_p] * 8 +
                           [C.POINTER(SolveStats), _p]),
    "ryo_solve_arrays_get": (_i, [_p, C.POINTER(SolveArrays)]),
    "ryo_engine_params_default": (None, [C.POINTER(EngineParams)]),
    "ryo_engine_create": (_i, [_p, C.POINTER(EngineParams), C.POINTER(C.c_void_p)]),
    "ryo_engine_destroy": (None, [_p]),
    "ryo_engine_last_error": (C.c_char_p, [_p]),
    "ryo_engine_submit": (_i, [_p, C.POINTER(EngineRequest)]),
    "ryo_engine_step": (_i, [_p, C.POINTER(EngineStepInfo), _p]),
    "ryo_engine_poll": (_i, [_p, C.POINTER(EngineResult), _i, C.POINTER(C.c_int)]),
    "ryo_engine_status": (_i, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "ryo_ewald_targets_f64": (_i, [_p, _p, _sz] + [_p] * 4 + [_sz, C.c_double, C.POINTER(EwaldSettings), C.c_double]
                              + [_p] * 5),
    "ryo_compute_group_splits_f32": (_i, [_p, _u32, _u32] + [_p] * 5 + [_i, _p, C.POINTER(BoxF32), _u, C.c_float,
                                                                      C.c_float, _p, _u32, C.POINTER(C.c_uint32), _p]),
    "ryo_solve_targets_f32": (_i, [_p] * 6 + [_sz] + [_p] * 4 + [C.POINTER(SolveStats), _p]),
    "ryo_solve_batch_f32": (_i, [_p, C.POINTER(SolveParams), C.POINTER(System), _i] + [_p] * 8 + [_sz] + [_p] * 7
                            + [C.POINTER(SolveStats), _p]),
    "ryo_kernel_launches": (C.c_uint64, []),
    "ryo_measure_peaks": (_i, [_p, C.POINTER(_d), _p]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"ryoanji_b200: {path} is missing; build it with `python -m ryoanji_b200.build` "
                          "(there is no CPU fallback)")
    handle = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


class _LazyLib:
    """loads the shared library on first use, so that the build module can run before it exists"""

    _handle = None

    def __getattr__(self, name):
        if _LazyLib._handle is None:
            _LazyLib._handle = load()
        return getattr(_LazyLib._handle, name)

    def loaded(self):
        if _LazyLib._handle is None:
            _LazyLib._handle = load()
        return _LazyLib._handle


lib = _LazyLib()


class _CudaArray:
    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


_TYPESTR = {torch.int32: "<i4", torch.int64: "<i8", torch.float32: "<f4", torch.float64: "<f8"}


def wrap_device(ptr, count: int, dtype, device) -> torch.Tensor:
    """a torch view of library-owned device memory (valid until the owner reallocates it)"""
    if not ptr or count == 0:
        return torch.empty(0, dtype=dtype, device=device)
    return torch.as_tensor(_CudaArray(ptr, count, _TYPESTR[dtype]), device=device)
