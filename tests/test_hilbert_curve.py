"""The keys trace a Hilbert curve: properties from the reference's own Hilbert tests, on the oracle (CPU) and on the
library's key kernel (GPU).

- cstone/test/unit/sfc/hilbert.cpp:259-293: the level-1 octants of the cells (0,1,1), (0,1,0) and (1,1,1) carry
  the octal digits 2, 3 and 5;
- hilbert.cpp:120-145: consecutive keys are face neighbours (checked there at octant crossings, here for every pair
  of consecutive cells of a level);
- hilbert.cpp:150-182: decoding a key gives back its cell.
"""
import numpy as np
import pytest

UNIT = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
MAX_LEVEL = 21


def _cells(level):
    s = 1 << level
    i = np.arange(s)
    gx, gy, gz = (a.ravel() for a in np.meshgrid(i, i, i, indexing="ij"))
    centre = lambda g: ((g + 0.5) / s).astype(np.float32)  # noqa: E731
    return gx, gy, gz, centre(gx), centre(gy), centre(gz)


def _check_curve(keys, gx, gy, gz, level):
    prefix = keys >> np.uint64(3 * (MAX_LEVEL - level))
    assert np.array_equal(np.sort(prefix), np.arange(8 ** level, dtype=np.uint64))  # one cell per key prefix
    o = np.argsort(prefix)
    step = np.abs(np.diff(gx[o])) + np.abs(np.diff(gy[o])) + np.abs(np.diff(gz[o]))
    assert (step == 1).all()


def test_level_one_digits(oracle):
    for cell, digit in (((0, 0, 0), 0), ((0, 1, 1), 2), ((0, 1, 0), 3), ((1, 1, 1), 5)):
        x, y, z = (np.array([(c + 0.5) / 2], np.float32) for c in cell)
        assert int(oracle.sfc_keys(x, y, z, UNIT)[0]) >> 60 == digit, cell


def test_oracle_curve_is_continuous_and_decodes(oracle):
    level = 4
    gx, gy, gz, x, y, z = _cells(level)
    keys = oracle.sfc_keys(x, y, z, UNIT)
    _check_curve(keys, gx, gy, gz, level)
    bits = oracle.box_dim_bits(UNIT)
    w = 1 << (MAX_LEVEL - level)
    for k in range(0, len(keys), 17):
        box = oracle.hilbert_ibox(keys[k], level, bits)
        assert tuple(box) == (gx[k] * w, (gx[k] + 1) * w, gy[k] * w, (gy[k] + 1) * w, gz[k] * w, (gz[k] + 1) * w)


@pytest.mark.gpu
def test_gpu_curve_is_continuous_and_equals_oracle(oracle):
    """every cell of level 6, keyed by both of the library's key kernels: the bitwise encoder behind
    ryo_compute_sfc_keys_f32, and the state-table kernel of the solve (cubic boxes), seen through the solve's sorted
    keys and sorted positions"""
    import torch
    import ryoanji_b200 as ryo
    level = 6
    gx, gy, gz, x, y, z = _cells(level)
    ref = oracle.sfc_keys(x, y, z, UNIT)
    dev = [torch.from_numpy(a).cuda() for a in (x, y, z)]
    keys = ryo.compute_sfc_keys(*dev, ryo.Box.cube(0.0, 1.0)).cpu().numpy().view(np.uint64)
    assert np.array_equal(keys, ref)
    _check_curve(keys, gx, gy, gz, level)

    n = len(x)
    ctx = ryo.Context(0)
    m = torch.full((n,), 1.0 / n, device="cuda")
    h = torch.full((n,), 1e-3, device="cuda")
    out = [torch.empty(n, device="cuda") for _ in range(4)]
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    ryo.solve(*dev, m, h, *out, params=ryo.SolveParams(box=ryo.Box.cube(0.0, 1.0)), order=order, ctx=ctx)
    sorted_keys = ryo.solve_arrays(ctx)["sortedKeys"].cpu().numpy().view(np.uint64)
    assert np.array_equal(sorted_keys, np.sort(ref))
    o = order.cpu().numpy()
    assert np.array_equal(ref[o], sorted_keys)
    s = 1 << level
    cx, cy, cz = ((t.cpu().numpy() * s).astype(np.int64) for t in dev)  # the positions, now in key order
    assert np.array_equal(cx, gx[o]) and np.array_equal(cy, gy[o]) and np.array_equal(cz, gz[o])
    step = np.abs(np.diff(cx)) + np.abs(np.diff(cy)) + np.abs(np.diff(cz))
    assert (step == 1).all()
