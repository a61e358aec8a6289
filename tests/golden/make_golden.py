"""Writes the golden fixtures of tests/golden/ by running the reference's own CPU code.

Run in a checkout where the reference tree exists (it is compiled by oracle/Makefile into oracle/_ref):

    python tests/golden/make_golden.py

Each case stores seeded inputs and the reference's outputs of: computeSfcKeys, sort_by_key, computeOctree,
updateInternalTree, the CPU upsweep (centres, multipoles, MAC radii), computeGravity, directSum and
computeGravityEwald. The fixtures pin the restated oracle (tests/test_oracle_golden.py), which then checks the GPU.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from pyoracle import Oracle, build  # noqa: E402


def inputs(kind: str, n: int, seed: int):
    rng = np.random.default_rng(seed)
    if kind == "cube":
        x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
        box = [-1, 1, -1, 1, -1, 1]
    elif kind == "gauss":
        x, y, z = (np.clip(rng.normal(0, 0.15, n), -1, 1) for _ in range(3))
        box = [-1, 1, -1, 1, -1, 1]
    elif kind == "clumps":
        c = rng.uniform(-0.9, 0.9, (6, 3))
        idx = rng.integers(0, 6, n)
        p = np.clip(c[idx] + rng.normal(0, 1e-3, (n, 3)), -1, 1)
        x, y, z = p.T
        box = [-1, 1, -1, 1, -1, 1]
    elif kind == "mixd":
        x, y, z = rng.uniform(0, 4, n), rng.uniform(0, 1, n), rng.uniform(0, 0.3, n)
        box = [0, 4, 0, 1, 0, 0.3]
    elif kind == "periodic":
        x, y, z = (rng.uniform(0, 1, n) for _ in range(3))
        box = [0, 1, 0, 1, 0, 1]
    else:
        raise ValueError(kind)
    m = rng.uniform(0.5, 1.5, n) / n
    h = np.full(n, 0.01)
    f = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    return f(x), f(y), f(z), f(m), f(h), np.asarray(box, np.float32)


CASES = [("cube", 4096, 1, 16), ("gauss", 4096, 2, 32), ("clumps", 2048, 3, 8), ("mixd", 2048, 4, 16),
         ("periodic", 1024, 5, 16)]


def make_case(ref: Oracle, kind: str, n: int, seed: int, bucket: int, theta: float = 0.5):
    x, y, z, m, h, box = inputs(kind, n, seed)
    out = dict(x=x, y=y, z=z, m=m, h=h, box=box, bucket=np.int32(bucket), theta=np.float32(theta))
    keys = ref.sfc_keys(x, y, z, box)
    skeys, order = ref.sort_keys(keys)
    leaves, counts = ref.octree_leaves(skeys, bucket)
    tree = ref.octree_link(leaves)
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    xs, ys, zs, ms, hs = (a[order] for a in (x, y, z, m, h))
    centers, mp = ref.upsweep(xs, ys, zs, ms, layout, tree, theta, box)
    out.update(keys=keys, sorted_keys=skeys, order=order, leaves=leaves, counts=counts, layout=layout,
               centers=centers, multipoles=mp, bits=ref.box_dim_bits(box))
    for k in ("prefixes", "childOffsets", "parents", "levelRange", "internalToLeaf", "leafToInternal"):
        out["tree_" + k] = tree[k]
    if n % 16 == 0 and kind != "periodic":
        u, pot, ax, ay, az = ref.gravity_cpu(tree, centers, mp, layout, xs, ys, zs, hs, ms, box, G=1.0)
        out.update(grav_u=np.float64(u), grav_pot=pot, grav_ax=ax, grav_ay=ay, grav_az=az)
    if kind != "periodic" and n <= 4096:
        d = ref.direct_all_ref(*(a.astype(np.float64) for a in (xs, ys, zs, hs, ms)), G=1.0)
        out.update(direct_pot=d[0], direct_ax=d[1], direct_ay=d[2], direct_az=d[3])
    if kind == "periodic":
        root_c = centers[0, :3].astype(np.float64)
        mroot = mp[0].astype(np.float64)
        u, pot, ax, ay, az = ref.ewald(root_c, mroot, *(a.astype(np.float64) for a in (xs, ys, zs, ms)),
                                       box.astype(np.float64), G=1.0)
        out.update(ewald_u=np.float64(u), ewald_pot=pot, ewald_ax=ax, ewald_ay=ay, ewald_az=az)
    return out


def main():
    build(reference=True)
    ref = Oracle(reference=True)
    for kind, n, seed, bucket in CASES:
        data = make_case(ref, kind, n, seed, bucket)
        np.savez_compressed(os.path.join(HERE, f"case_{kind}_{n}.npz"), **data)
        print(kind, n, "leaves", len(data["counts"]))
    # known answers quoted by the reference's unit tests
    h1 = np.sqrt(3) / 2 - 0.001
    h2 = np.sqrt(3) / 2 + 0.001
    kv = dict(
        p2p_base=np.array([-0.76980035891950138, 0.17106674642655587, 0.17106674642655587, 0.17106674642655587]),
        p2p_soft=np.array([-0.7678049688481372, 0.1704016164027678, 0.1704016164027678, 0.1704016164027678]),
        p2p_h=np.array([h1, h2]),
        ewald_single=np.array([1.4717464459658256, 0.7358732229829128]),
        fixed_groups=np.array([4, 12, 20, 28, 34]),
    )
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **kv)
    print("known answers written")


if __name__ == "__main__":
    main()
