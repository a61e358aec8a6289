"""The sort entry point without temporary-storage argument (ryo_sort_by_key_static), called through the C ABI.

Its keys and payload must equal those of ryo_sort_by_key, bit for bit, on two calls in a row (the second call reuses
the fixed scratch the first one left behind). This file sorts last so the check also runs after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 24
ERR_CAPACITY = 6


def _lib():
    import ryoanji_b200 as ryo
    return ryo.lib


def _p(t):
    return C.c_void_p(t.data_ptr())


def sort_with_caller_storage(keys, vals):
    lib = _lib()
    n = keys.numel()
    kb, vb = torch.empty_like(keys), torch.empty_like(vals)
    tmp = torch.empty(int(lib.ryo_sort_by_key_temp_bytes(C.c_size_t(n))), dtype=torch.uint8, device=keys.device)
    st = lib.ryo_sort_by_key(_p(keys), _p(vals), C.c_size_t(n), _p(kb), _p(vb), _p(tmp), C.c_size_t(tmp.numel()),
                             None)
    assert st == 0, lib.ryo_ctx_last_error(None)


def sort_static(keys, vals):
    lib = _lib()
    kb, vb = torch.empty_like(keys), torch.empty_like(vals)
    return lib.ryo_sort_by_key_static(_p(keys), _p(vals), C.c_size_t(keys.numel()), _p(kb), _p(vb), None)


def make_keys(n, seed):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 2 ** 63, n, dtype=np.int64)
    k[rng.integers(0, n, n // 4 + 1)] = k[n // 2]  # runs of equal keys test stability
    return torch.from_numpy(k).cuda()


@pytest.mark.parametrize("n", [1, 3073, 200003, MAX_KEYS])
def test_static_sort_matches_caller_storage_sort_twice(n):
    for call, seed in enumerate((n, n + 1)):
        src = make_keys(n, seed)
        ka, va = src.clone(), torch.arange(n, dtype=torch.int32, device="cuda")
        kb, vb = src.clone(), va.clone()
        sort_with_caller_storage(ka, va)
        st = sort_static(kb, vb)
        assert st == 0, (call, _lib().ryo_ctx_last_error(None))
        torch.cuda.synchronize()
        assert torch.equal(ka, kb), call
        assert torch.equal(va, vb), call
    if n <= 200003:
        k = src.cpu().numpy()
        order = np.argsort(k, kind="stable")
        assert np.array_equal(kb.cpu().numpy(), k[order])
        assert np.array_equal(vb.cpu().numpy(), order.astype(np.int32))


def test_static_sort_rejects_too_many_keys_and_leaves_data():
    n = MAX_KEYS + 1
    keys = make_keys(n, 3)
    before = keys.clone()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    assert sort_static(keys, vals) == ERR_CAPACITY
    assert b"RYO_SORT_STATIC_MAX_KEYS" in _lib().ryo_ctx_last_error(None)
    assert torch.equal(keys, before)
    # the entry point still works after the rejection
    small = make_keys(5000, 4)
    ref, rv = small.clone(), torch.arange(5000, dtype=torch.int32, device="cuda")
    sv = rv.clone()
    sort_with_caller_storage(ref, rv)
    assert sort_static(small, sv) == 0
    assert torch.equal(ref, small) and torch.equal(rv, sv)


def test_static_sort_empty_is_a_no_op():
    lib = _lib()
    assert lib.ryo_sort_by_key_static(None, None, C.c_size_t(0), None, None, None) == 0
