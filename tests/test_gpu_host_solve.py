"""Solve from and to host memory (ryo_solve_host_f32): the same results as the device solve.

Inputs come from pinned host tensors and are left unchanged; outputs (sorted positions, order, potential and
acceleration in SFC order) land in host tensors.
- Pinned output arrays: the traversal of an open system stores its results straight into them. It is the device
  solve's launch, so the results are bit-identical.
- Pageable output arrays: the traversal runs in chunks of groups whose results download while the next chunk runs.
  Every group is computed by the same kernel code as in one launch, so the results are bit-identical, except for
  groups split over several warps, whose part count may differ (rounding).
"""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def _compare(pset, params, exact, pinned_out=True):
    import ryoanji_b200 as ryo
    n = pset.n
    hin = [_pinned(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h)]
    before = [t.clone() for t in hin]
    hout = [torch.empty(n).pin_memory() if pinned_out else torch.empty(n) for _ in range(4)]
    hxyz = [torch.empty(n).pin_memory() for _ in range(3)]
    hord = torch.empty(n, dtype=torch.int32).pin_memory()
    ctx = ryo.Context()
    rh = ryo.solve_host(*hin, *hout, params=params, sorted_xyz=hxyz, order=hord, ctx=ctx)
    for a, b in zip(hin, before):
        assert torch.equal(a, b)  # inputs untouched

    d = [t.cuda() for t in hin]
    dout = [torch.empty(n, device="cuda") for _ in range(4)]
    dord = torch.empty(n, dtype=torch.int32, device="cuda")
    rd = ryo.solve(*d, *dout, params=params, order=dord, ctx=ctx)
    assert torch.equal(hord, dord.cpu())
    for a, b in zip(hxyz, d[:3]):
        assert torch.equal(a, b.cpu())
    assert (rh.sum_p2p, rh.max_p2p, rh.sum_m2p, rh.max_m2p) == (rd.sum_p2p, rd.max_p2p, rd.sum_m2p, rd.max_m2p)
    for a, b in zip(hout, dout):
        b = b.cpu()
        if exact:
            assert torch.equal(a, b)
        else:
            scale = b.abs().max()
            assert float((a - b).abs().max()) <= 1e-6 * float(scale)
    assert rh.potential_energy == pytest.approx(rd.potential_energy, rel=1e-9 if exact else 1e-6)
    return rh


def test_host_solve_equals_device_solve_cube():
    import ryoanji_b200 as ryo
    _compare(ds.uniform_cube(300000, seed=3), ryo.SolveParams(theta=0.5), exact=True)


def test_host_solve_equals_device_solve_with_split_groups():
    import ryoanji_b200 as ryo
    pset = ds.plummer(100000, seed=1, velocities=False)
    r = _compare(pset, ryo.SolveParams(theta=0.5), exact=True)
    assert r.max_p2p > 16384  # the sparse outskirts took the split path
    _compare(pset, ryo.SolveParams(theta=0.5), exact=False, pinned_out=False)


def test_host_solve_into_pageable_outputs():
    import ryoanji_b200 as ryo
    pset = ds.uniform_cube(300000, seed=3)
    _compare(pset, ryo.SolveParams(theta=0.5), exact=True, pinned_out=False)
    _compare(pset, ryo.SolveParams(theta=0.5, group_tolerance=2.0), exact=True, pinned_out=False)
    _compare(pset, ryo.SolveParams(theta=0.5, group_tolerance=2.0), exact=True)  # spatial groups, stored directly


def test_host_solve_periodic_and_small():
    import ryoanji_b200 as ryo
    p = ds.periodic_box(20000, seed=6, eps=0.002)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    _compare(p, ryo.SolveParams(theta=0.5, box=box), exact=True)
    _compare(ds.uniform_cube(100, seed=4, eps=0.01), ryo.SolveParams(theta=0.5), exact=True)  # fewer groups than chunks


def test_host_solve_rejects_device_tensors():
    import ryoanji_b200 as ryo
    x = torch.zeros(16, device="cuda")
    with pytest.raises(ValueError):
        ryo.solve_host(x, x, x, x, x, x, x, x, x)


def test_host_solve_into_registered_outputs():
    """outputs in host memory page-locked by cudaHostRegister (default flags) rather than allocated pinned"""
    import ryoanji_b200 as ryo
    cudart = torch._C._cudart
    pset = ds.uniform_cube(200000, seed=5)
    n = pset.n
    outs = [np.empty(n, np.float32) for _ in range(4)]
    registered = []
    try:
        for a in outs:
            assert int(cudart.cudaHostRegister(a.ctypes.data, a.nbytes, 0)) == 0
            registered.append(a)
        hin = [_pinned(a) for a in (pset.x, pset.y, pset.z, pset.m, pset.h)]
        hout = [torch.from_numpy(a) for a in outs]
        hord = torch.empty(n, dtype=torch.int32)
        ctx = ryo.Context()
        params = ryo.SolveParams(theta=0.5)
        ryo.solve_host(*hin, *hout, params=params, order=hord, ctx=ctx)
        d = [t.cuda() for t in hin]
        dout = [torch.empty(n, device="cuda") for _ in range(4)]
        ryo.solve(*d, *dout, params=params, ctx=ctx)
        for a, b in zip(hout, dout):
            assert torch.equal(a, b.cpu())
    finally:
        for a in registered:
            cudart.cudaHostUnregister(a.ctypes.data)


def test_host_solve_signed_masses_mdq():
    """monopole + dipole + quadrupole expansions of signed masses: the host solve equals the device solve"""
    import ryoanji_b200 as ryo
    p = ds.gaussian(60000, seed=35, sigma=0.2)
    m = np.full(p.n, 1.0 / p.n)
    m[1::2] *= -1.0
    p.m = m.astype(np.float32)
    p.h = np.full(p.n, 0.002, np.float32)
    params = ryo.SolveParams(theta=0.5, box=ryo.Box.cube(-1.0, 1.0), multipole="mdq")
    _compare(p, params, exact=True)
    # 938 groups: the split threshold falls with the group count, and the chunked launches split groups into other
    # part counts than one launch does
    _compare(p, params, exact=False, pinned_out=False)
