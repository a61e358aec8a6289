"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU oracle and of the reference's own CPU path.

``Oracle()`` loads the restated oracle (oracle/_build/libryo_oracle.so); ``Oracle(reference=True)`` loads the
reference's CPU code behind the same interface (oracle/_ref/libryo_ref.so, built only where the reference tree is
present). Only tests, the smoke check and bench.py's cpu_baseline leg use this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libryo_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libryo_ref.so")

_p = C.c_void_p
_sz = C.c_size_t


def build(reference: bool = False) -> None:
    """Compile the oracle (and, if asked and possible, the reference wrapper) with oracle/Makefile."""
    target = ["all"] if reference else ["oracle"]
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def timing_builds() -> list[tuple[str, str]]:
    """the builds of the reference's CPU path this host can run, with their compiler flags: the -O3 -fopenmp builds
    for the vector ISAs the host supports (oracle/Makefile target reffast) and the parity build"""
    flags = _cpu_flags()
    need = {"v4": {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}, "v3": {"avx2", "fma", "bmi2", "movbe"}}
    out = []
    for level in ("v4", "v3"):
        path = os.path.join(HERE, "_ref", f"libryo_ref_fast_{level}.so")
        if need[level] <= flags and os.path.exists(path):
            out.append((path, f"g++ -O3 -march=x86-64-{level} -fopenmp (default FP contraction)"))
    out.append((REF_SO, "g++ -O3 -fopenmp -ffp-contract=off (x86-64 baseline)"))
    return out


def _ptr(a):
    return a.ctypes.data_as(_p) if a is not None else None


class Oracle:
    """The CPU path with one Python interface for both the restatement (orc_*) and the reference (ref_*)."""

    def __init__(self, reference: bool = False, library: str | None = None):
        """library (with reference=True) loads another build of the reference's CPU path (timing_builds) in place of
        the parity build; its results follow that build's FP contraction and are for timing only"""
        path = REF_SO if reference else ORACLE_SO
        if reference and library:
            path = library
        if not os.path.exists(path):
            build(reference)
        self.reference = reference
        self.lib = C.CDLL(path)
        self.pre = "ref_" if reference else "orc_"

    def _f(self, name, restype=None):
        fn = getattr(self.lib, self.pre + name)
        fn.restype = restype
        return fn

    # ---- keys
    def sfc_keys(self, x, y, z, box6):
        dt = x.dtype
        keys = np.zeros(len(x), np.uint64)
        box = np.asarray(box6, dt)
        name = "sfc_keys_f32" if dt == np.float32 else "sfc_keys_f64"
        self._f(name)(_ptr(x), _ptr(y), _ptr(z), _sz(len(x)), _ptr(box), _ptr(keys))
        return keys

    def box_dim_bits(self, box6):
        bits = np.zeros(3, np.uint32)
        self._f("box_dim_bits_f32")(_ptr(np.asarray(box6, np.float32)), _ptr(bits))
        return bits

    def hilbert_ibox(self, key, level, bits):
        out = np.zeros(6, np.int32)
        self._f("hilbert_ibox")(C.c_uint64(int(key)), C.c_uint(level), C.c_uint(int(bits[0])), C.c_uint(int(bits[1])),
                                C.c_uint(int(bits[2])), _ptr(out))
        return out

    def sort_keys(self, keys):
        k = np.ascontiguousarray(keys, np.uint64).copy()
        order = np.zeros(len(k), np.uint32)
        self._f("sort_keys")(_ptr(k), _ptr(order), _sz(len(k)))
        return k, order

    # ---- tree
    def octree_leaves(self, sorted_keys, bucket):
        k = np.ascontiguousarray(sorted_keys, np.uint64)
        fn = self._f("octree_leaves", C.c_long)
        n = fn(_ptr(k), _sz(len(k)), C.c_uint(bucket), None, None, C.c_long(0))
        leaves = np.zeros(n + 1, np.uint64)
        counts = np.zeros(n, np.uint32)
        fn(_ptr(k), _sz(len(k)), C.c_uint(bucket), _ptr(leaves), _ptr(counts), C.c_long(n))
        return leaves, counts

    def octree_link(self, leaves):
        nl = len(leaves) - 1
        ni = (nl - 1) // 7
        nn = nl + ni
        t = dict(
            prefixes=np.zeros(nn, np.uint64),
            childOffsets=np.zeros(nn, np.int32),
            parents=np.zeros(max(1, (nn - 1) // 8), np.int32),
            levelRange=np.zeros(23, np.int32),
            internalToLeaf=np.zeros(nn, np.int32),
            leafToInternal=np.zeros(nn, np.int32),
        )
        self._f("octree_link")(_ptr(np.ascontiguousarray(leaves, np.uint64)), C.c_int(nl), _ptr(t["prefixes"]),
                               _ptr(t["childOffsets"]), _ptr(t["parents"]), _ptr(t["levelRange"]),
                               _ptr(t["internalToLeaf"]), _ptr(t["leafToInternal"]))
        t.update(numLeaves=nl, numInternal=ni, numNodes=nn)
        return t

    # ---- upsweep
    def upsweep(self, x, y, z, m, layout, tree, theta, box6, mode=0):
        nn = tree["numNodes"]
        centers = np.zeros((nn, 4), np.float32)
        mp = np.zeros((nn, 8), np.float32)
        l2i = np.ascontiguousarray(tree["leafToInternal"][tree["numInternal"]:])
        args = [_ptr(x), _ptr(y), _ptr(z), _ptr(m)]
        if self.reference:
            assert mode == 0, "the reference upsweep is float only"
            self._f("upsweep_f32")(*args, _sz(len(x)), C.c_int(tree["numLeaves"]), _ptr(layout), _ptr(l2i),
                                   _ptr(tree["childOffsets"]), _ptr(tree["levelRange"]), _ptr(tree["prefixes"]),
                                   C.c_int(nn), C.c_float(theta), _ptr(np.asarray(box6, np.float32)), _ptr(centers),
                                   _ptr(mp))
        else:
            self._f("upsweep_f32")(C.c_int(mode), *args, C.c_int(tree["numLeaves"]), _ptr(layout), _ptr(l2i),
                                   _ptr(tree["childOffsets"]), _ptr(tree["levelRange"]), _ptr(tree["prefixes"]),
                                   C.c_int(nn), C.c_float(theta), _ptr(np.asarray(box6, np.float32)), _ptr(centers),
                                   _ptr(mp))
        return centers, mp

    def upsweep_mdq(self, x, y, z, m, layout, tree, theta, box6):
        """the reference CPU upsweep with CartesianMDQpole multipoles (12 floats per node)"""
        assert self.reference
        nn = tree["numNodes"]
        centers = np.zeros((nn, 4), np.float32)
        mp = np.zeros((nn, 12), np.float32)
        l2i = np.ascontiguousarray(tree["leafToInternal"][tree["numInternal"]:])
        self._f("upsweep_mdq_f32")(_ptr(x), _ptr(y), _ptr(z), _ptr(m), _sz(len(x)), C.c_int(tree["numLeaves"]),
                                   _ptr(layout), _ptr(l2i), _ptr(tree["childOffsets"]), _ptr(tree["levelRange"]),
                                   _ptr(tree["prefixes"]), C.c_int(nn), C.c_float(theta),
                                   _ptr(np.asarray(box6, np.float32)), _ptr(centers), _ptr(mp))
        return centers, mp

    # ---- gravity
    def gravity_cpu(self, tree, centers, mp, layout, x, y, z, h, m, box6, G=1.0, numShells=0, periodic=False):
        n = len(x)
        pot, ax, ay, az = (np.zeros(n, np.float32) for _ in range(4))
        head = [_ptr(tree["childOffsets"]), _ptr(tree["parents"]), _ptr(tree["internalToLeaf"]), _ptr(centers),
                _ptr(mp), _ptr(layout), C.c_int(tree["numLeaves"]), _ptr(x), _ptr(y), _ptr(z), _ptr(h), _ptr(m),
                _ptr(np.asarray(box6, np.float32))]
        if self.reference:
            u = self._f("gravity_cpu_f32", C.c_double)(*head, C.c_int(int(periodic)), C.c_float(G), C.c_int(numShells),
                                                        _ptr(pot), _ptr(ax), _ptr(ay), _ptr(az))
        else:
            u = self._f("gravity_cpu_f32", C.c_double)(*head, C.c_float(G), C.c_int(numShells), _ptr(pot), _ptr(ax),
                                                        _ptr(ay), _ptr(az))
        return u, pot, ax, ay, az

    def traverse_rule(self, group_start, group_end, x, y, z, h, m, tree, layout, centers, mp, init_node=1,
                      numShells=0, boxL=(0.0, 0.0, 0.0), evaluate=False):
        assert not self.reference
        ng = len(group_start)
        m2p = np.zeros(ng, np.uint32)
        p2p = np.zeros(ng, np.uint32)
        acc = np.zeros((len(x), 4), np.float64) if evaluate else None
        gs = np.ascontiguousarray(group_start, np.uint32)
        ge = np.ascontiguousarray(group_end, np.uint32)
        self._f("traverse_rule")(C.c_int(ng), _ptr(gs), _ptr(ge), _ptr(x), _ptr(y), _ptr(z), _ptr(h), _ptr(x),
                                 _ptr(y), _ptr(z), _ptr(m), _ptr(h), _ptr(tree["childOffsets"]),
                                 _ptr(tree["internalToLeaf"]), _ptr(layout), _ptr(centers), _ptr(mp),
                                 C.c_int(init_node), C.c_int(numShells), _ptr(np.asarray(boxL, np.float32)), _ptr(m2p),
                                 _ptr(p2p), _ptr(acc))
        return m2p, p2p, acc

    def direct(self, x, y, z, h, m, targets, G=1.0, boxL=(0.0, 0.0, 0.0), numShells=0):
        assert not self.reference
        t = np.ascontiguousarray(targets, np.int64)
        out = [np.zeros(len(t), np.float64) for _ in range(4)]
        self._f("direct_f64")(_ptr(x), _ptr(y), _ptr(z), _ptr(h), _ptr(m), _sz(len(x)), _ptr(t), _sz(len(t)),
                              C.c_double(G), _ptr(np.asarray(boxL, np.float64)), C.c_int(numShells), *map(_ptr, out))
        return out  # pot, ax, ay, az

    def direct_all_ref(self, x, y, z, h, m, G=1.0, boxL=(0.0, 0.0, 0.0), numShells=0):
        """the reference's own directSum (all targets), double"""
        assert self.reference
        n = len(x)
        out = [np.zeros(n, np.float64) for _ in range(4)]  # ax, ay, az, pot
        self._f("direct_f64")(_ptr(x), _ptr(y), _ptr(z), _ptr(h), _ptr(m), C.c_uint(n), C.c_float(G),
                              _ptr(np.asarray(boxL, np.float64)), C.c_int(numShells), *map(_ptr, out))
        ax, ay, az, pot = out
        return pot, ax, ay, az

    def p2p(self, ti, sj, mj, hi, hj, acc=None):
        a = np.zeros(4) if acc is None else np.array(acc, np.float64)
        self._f("p2p_f64")(_ptr(np.asarray(ti, np.float64)), _ptr(np.asarray(sj, np.float64)), C.c_double(mj),
                           C.c_double(hi), C.c_double(hj), _ptr(a))
        return a

    def p2m(self, x, y, z, m):
        c = np.zeros(4)
        q = np.zeros(8)
        self._f("p2m_f64")(_ptr(x), _ptr(y), _ptr(z), _ptr(m), C.c_uint(len(x)), _ptr(c), _ptr(q))
        return c, q

    def m2p(self, target, center, quad, acc=None):
        a = np.zeros(4) if acc is None else np.array(acc, np.float64)
        self._f("m2p_f64")(_ptr(np.asarray(target, np.float64)), _ptr(np.asarray(center, np.float64)),
                           _ptr(np.asarray(quad, np.float64)), _ptr(a))
        return a

    def ewald(self, root_center, mroot, x, y, z, m, box6, G=1.0, replica_shells=1, lcut=2.6, hcut=2.8,
              alpha_scale=2.0, small_r=3.0e-3):
        n = len(x)
        dt = x.dtype
        pot, ax, ay, az = (np.zeros(n, dt) for _ in range(4))
        rc = np.asarray(root_center, dt)
        mr = np.asarray(mroot, dt)
        box = np.asarray(box6, dt)
        if self.reference:
            name = "ewald_f32" if dt == np.float32 else "ewald_f64"
            u = self._f(name, C.c_double)(_ptr(rc), _ptr(mr), _ptr(x), _ptr(y), _ptr(z), _ptr(m), C.c_uint(n),
                                          _ptr(box), C.c_float(G), _ptr(pot), _ptr(ax), _ptr(ay), _ptr(az),
                                          C.c_int(replica_shells), C.c_double(lcut), C.c_double(hcut),
                                          C.c_double(alpha_scale), C.c_double(small_r))
        else:
            assert dt == np.float64
            u = self._f("ewald_f64", C.c_double)(_ptr(rc), _ptr(mr), _ptr(x), _ptr(y), _ptr(z), _ptr(m), _sz(n),
                                                 _ptr(box), C.c_double(G), _ptr(pot), _ptr(ax), _ptr(ay), _ptr(az),
                                                 C.c_int(replica_shells), C.c_double(lcut), C.c_double(hcut),
                                                 C.c_double(alpha_scale), C.c_double(small_r))
        return u, pot, ax, ay, az

    # ---- monopole + dipole + quadrupole (same names for the restatement and the reference wrapper)
    def mdq_p2m(self, x, y, z, m):
        c = np.zeros(4)
        q = np.zeros(12)
        self._f("mdq_p2m_f64")(*(_ptr(np.ascontiguousarray(a, np.float64)) for a in (x, y, z, m)),
                               C.c_uint(len(x)), _ptr(c), _ptr(q))
        return c, q

    def mdq_m2m(self, centers, mdqs, out_center):
        out = np.zeros(12)
        self._f("mdq_m2m_f64")(C.c_int(len(centers)), _ptr(np.ascontiguousarray(centers, np.float64)),
                               _ptr(np.ascontiguousarray(mdqs, np.float64)),
                               _ptr(np.ascontiguousarray(out_center, np.float64)), _ptr(out))
        return out

    def mdq_m2p(self, target, center, mdq):
        acc = np.zeros(4)
        self._f("mdq_m2p_f64")(_ptr(np.ascontiguousarray(target, np.float64)),
                               _ptr(np.ascontiguousarray(center, np.float64)),
                               _ptr(np.ascontiguousarray(mdq, np.float64)), _ptr(acc))
        return acc

    # ---- spatial target groups (restatement only: the reference's version is device code)
    def find_splits(self, pos4, dist_crit_sq):
        """split bits of one window of targets (rows x, y, z, w)"""
        assert not self.reference
        pos = np.ascontiguousarray(pos4, np.float64)
        return int(self._f("find_splits_f64", C.c_uint64)(_ptr(pos), C.c_int(len(pos)), C.c_double(dist_crit_sq)))

    def make_splits(self, mask, group_size=64):
        assert not self.reference
        out = np.zeros(group_size + 1, np.uint32)
        k = self._f("make_splits", C.c_int)(C.c_uint64(mask), C.c_int(group_size), _ptr(out))
        return out[:k]

    def group_splits(self, first, last, x, y, z, h, leaves, layout, box6, group_size=64, tol_factor=2.0,
                     extent_ratio=8.0):
        """(groups[numGroups + 1], counts per fixed window)"""
        assert not self.reference
        dt = x.dtype
        name = "group_splits_f32" if dt == np.float32 else "group_splits_f64"
        nl = len(leaves) - 1
        nw = (last - first + group_size - 1) // group_size
        counts = np.zeros(max(nw, 1), np.uint32)
        cap = last - first + 2
        groups = np.zeros(cap, np.uint32)
        hp = _ptr(np.ascontiguousarray(h, dt)) if h is not None else None
        ng = self._f(name, C.c_long)(C.c_uint32(first), C.c_uint32(last), _ptr(x), _ptr(y), _ptr(z), hp,
                                     _ptr(np.ascontiguousarray(leaves, np.uint64)), C.c_int(nl),
                                     _ptr(np.ascontiguousarray(layout, np.uint32)), _ptr(np.asarray(box6, dt)),
                                     C.c_int(group_size), C.c_float(tol_factor), C.c_float(extent_ratio),
                                     _ptr(counts), _ptr(groups), C.c_long(cap))
        return groups[:ng + 1].copy(), counts[:nw].copy()

    def ewald_single_particle_energy(self, m, N, L, G=1.0, alpha_scale=2.0):
        return self._f("ewald_single_particle_energy", C.c_double)(C.c_double(m), C.c_uint(N), C.c_double(L),
                                                                    C.c_double(G), C.c_double(alpha_scale))

    def solve(self, x, y, z, m, h, box6, bucket=64, theta=0.5, G=1.0):
        """the whole CPU path on copies of the inputs; returns (energy, sorted xyzmh, pot, ax, ay, az, seconds)"""
        xs, ys, zs, ms, hs = (np.array(a, np.float32) for a in (x, y, z, m, h))
        n = len(xs)
        pot, ax, ay, az = (np.zeros(n, np.float32) for _ in range(4))
        sec = np.zeros(3)
        u = self._f("solve_f32", C.c_double)(_ptr(xs), _ptr(ys), _ptr(zs), _ptr(ms), _ptr(hs), _sz(n),
                                             _ptr(np.asarray(box6, np.float32)), C.c_uint(bucket), C.c_float(theta),
                                             C.c_float(G), _ptr(pot), _ptr(ax), _ptr(ay), _ptr(az), _ptr(sec))
        return u, (xs, ys, zs, ms, hs), pot, ax, ay, az, sec
