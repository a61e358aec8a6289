"""The reference demo's flow written in the reference's spellings (tests/cpp/demo_flow.cpp, compiled against
ryoanji_b200/compat.hpp) runs on the GPU for the three type sets and gives exactly what the same steps give through
the Python API: the same readBhStats and accelerations bit for bit (one library, one order of work), and the same total
potential to the round-off of its atomic sum."""
import json
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _python_flow(xyz, dtype, mtype):
    import ryoanji_b200 as ryo
    n = xyz.shape[1]
    x, y, z = (torch.from_numpy(a.copy()).to("cuda", dtype) for a in xyz)
    m = torch.full((n,), 1.0 / n, dtype=mtype, device="cuda")
    h = torch.full((n,), 0.005, dtype=mtype, device="cuda")
    tb = ryo.TreeBuilder(64)
    box = ryo.Box(-1.0, 1.0, -1.0, 1.0, -1.0, 1.0)
    nn = tb.update(x, y, z, box)
    centers = torch.zeros(nn, 4, dtype=dtype, device="cuda")
    mp = torch.zeros(nn, 8, dtype=mtype, device="cuda")
    lr = tb.levelRange
    ryo.compute_leaf_source_center(x, y, z, m, tb.leafToInternal(), tb.layout(), centers)
    ryo.upsweep_centers(21, lr, tb.childOffsets(), centers)
    ryo.compute_leaf_multipoles(x, y, z, m, tb.leafToInternal(), tb.layout(), centers, mp)
    for level in range(20, 0, -1):
        ryo.upsweep_multipoles(lr[level], lr[level + 1], tb.childOffsets(), centers, mp)
    ryo.set_mac(tb.nodeKeys(), centers, 2.0, box)
    groups = ryo.compute_fixed_groups(0, n, 64)
    acc = [torch.zeros(n, dtype=mtype, device="cuda") for _ in range(4)]
    pot = ryo.traverse(groups, 1, x, y, z, m, h, x, y, z, m, h, tb.childOffsets(), tb.internalToLeaf(), tb.layout(),
                       centers, mp, 1.0, 0, None, *acc)
    return ryo.read_bh_stats()[:4], pot, np.stack([a.cpu().numpy().astype(np.float64) for a in acc[1:]])


def test_compat_demo_flow_equals_python_api(tmp_path):
    from ryoanji_b200._abi import LIB_PATH
    exe = tmp_path / "demo_flow"
    libdir = os.path.dirname(LIB_PATH)
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        os.path.join(ROOT, "tests", "cpp", "demo_flow.cpp"), "-o", str(exe), "-L", libdir,
                        "-lryoanji_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = 40000
    xyz = np.random.default_rng(41).uniform(-1, 1, (3, n)).astype(np.float32)
    inp = tmp_path / "bodies.bin"
    xyz.tofile(inp)
    run = subprocess.run([str(exe), str(inp), str(tmp_path / "acc")], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    lines = {d["set"]: d for d in (json.loads(l) for l in run.stdout.splitlines() if l.startswith("{"))}
    assert set(lines) == {"f32", "f64", "mixed"}
    for name, dtype, mtype in (("f32", torch.float32, torch.float32), ("f64", torch.float64, torch.float64),
                               ("mixed", torch.float64, torch.float32)):
        stats, pot, acc = _python_flow(xyz, dtype, mtype)
        assert lines[name]["stats"] == list(stats), (name, lines[name]["stats"], stats)
        # the total is an FP64 atomic sum over groups: its last bit depends on their order
        assert abs(lines[name]["potential"] - pot) <= 1e-13 * abs(pot), name
        cpp = np.fromfile(tmp_path / f"acc.{name}.bin", np.float64).reshape(3, n)
        assert np.array_equal(cpp, acc), name
    # the type sets differ only by precision: float-representable inputs give nearly the same field
    a32 = np.fromfile(tmp_path / "acc.f32.bin", np.float64).reshape(3, n)
    a64 = np.fromfile(tmp_path / "acc.f64.bin", np.float64).reshape(3, n)
    err = np.linalg.norm(a32 - a64, axis=0) / np.linalg.norm(a64, axis=0)
    assert np.percentile(err, 99) < 1e-4
