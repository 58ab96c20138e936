"""gs_stage_sort_noalloc: the tile-list sort for callers that cannot allocate
device memory (an application whose device memory all comes from its own
pool, or a frame loop that must not pay for cudaMalloc's device-wide
synchronisation).  Its scratch is a fixed array inside the library, so the
call allocates nothing; it must sort exactly like gs_stage_sort.

This file is collected last on purpose: a failure here does not hide the
rest of the suite in a run that stops at the first failure.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _noalloc(gs):
    f = gs.lib.gs_stage_sort_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int64, ctypes.c_int32] + [ctypes.c_void_p] * 4 + [ctypes.POINTER(ctypes.c_int32),
                                                                              ctypes.c_void_p]
    gs.lib.gs_stage_sort_noalloc_max_keys.restype = ctypes.c_int64
    gs.lib.gs_stage_sort_noalloc_error.restype = ctypes.c_char_p
    return f


def _keys(n, bits, seed):
    rng = np.random.default_rng(seed)
    tiles = rng.integers(0, 1 << (bits - 32), n).astype(np.uint64)
    depth = rng.integers(0, 1 << 20, n).astype(np.uint64)  # many equal keys
    return (tiles << np.uint64(32)) | depth, rng.permutation(n).astype(np.int32)


def _sort_noalloc(f, keys, vals, bits):
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.copy()).cuda()
    ka, va = torch.empty_like(k), torch.empty_like(v)
    torch.cuda.synchronize()
    sel = ctypes.c_int32(-1)
    free_before = torch.cuda.mem_get_info()[0]
    st = f(len(keys), bits, k.data_ptr(), v.data_ptr(), ka.data_ptr(), va.data_ptr(), ctypes.byref(sel), None)
    free_after = torch.cuda.mem_get_info()[0]
    assert st == 0
    out_k = (ka if sel.value else k).cpu().numpy().view(np.uint64)
    out_v = (va if sel.value else v).cpu().numpy()
    return out_k, out_v, free_before - free_after


def _sort_ctx(gs, ctx, keys, vals, bits):
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.copy()).cuda()
    ka, va = torch.empty_like(k), torch.empty_like(v)
    sel = gs.stage_sort(ctx, len(keys), bits, k, v, ka, va)
    torch.cuda.synchronize()
    return (ka if sel else k).cpu().numpy().view(np.uint64), (va if sel else v).cpu().numpy()


def test_sort_noalloc_matches_sort_two_calls_in_a_row(gs):
    f = _noalloc(gs)
    ctx = gs.Context(0)
    cases = [(1_000_003, 44, 1), (gs.lib.gs_stage_sort_noalloc_max_keys(), 51, 2)]
    # a first tiny call loads the library's kernels (lazy module loading may
    # take device memory once); the measured calls after it must take none
    wk, wv = _keys(1, 44, 0)
    _sort_noalloc(f, wk, wv, 44)
    consumed = []
    for n, bits, seed in cases:
        keys, vals = _keys(n, bits, seed)
        got_k, got_v, used = _sort_noalloc(f, keys, vals, bits)
        want_k, want_v = _sort_ctx(gs, ctx, keys, vals, bits)
        # integer sort: the results must be identical
        assert np.array_equal(got_k, want_k)
        assert np.array_equal(got_v, want_v)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_k, keys[order]) and np.array_equal(got_v, vals[order])
        consumed.append(used)
    # both calls run only already-loaded kernels: no device memory may move
    assert consumed == [0, 0]
    ctx.close()


def test_sort_noalloc_across_the_epoch_wrap(gs):
    """The look-back words are tagged with a 16-bit epoch that advances by
    one per pass; after about 0xFFFF / 8 calls of 64-bit keys it wraps and
    the words are cleared once.  Calls on both sides of the wrap sort
    exactly like numpy's stable sort."""
    f = _noalloc(gs)
    n, bits = 3000, 64
    rng = np.random.default_rng(9)
    keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * np.uint64(2)
    keys[::7] = keys[0]  # equal keys: the order of their values is checked too
    vals = rng.permutation(n).astype(np.int32)
    order = np.argsort(keys, kind="stable")
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.copy()).cuda()
    ka, va = torch.empty_like(k), torch.empty_like(v)
    sel = ctypes.c_int32(-1)
    calls = 0xFFFF // 8 + 3
    checked = 0
    for i in range(calls):
        k.copy_(torch.from_numpy(keys.view(np.int64)))
        v.copy_(torch.from_numpy(vals))
        assert f(n, bits, k.data_ptr(), v.data_ptr(), ka.data_ptr(), va.data_ptr(), ctypes.byref(sel), None) == 0
        if i < 2 or i >= calls - 4:
            out_k = (ka if sel.value else k).cpu().numpy().view(np.uint64)
            out_v = (va if sel.value else v).cpu().numpy()
            assert np.array_equal(out_k, keys[order]), i
            assert np.array_equal(out_v, vals[order]), i
            checked += 1
    assert checked == 6


def test_sort_noalloc_rejects_more_than_its_limit(gs):
    f = _noalloc(gs)
    limit = gs.lib.gs_stage_sort_noalloc_max_keys()
    sel = ctypes.c_int32(0)
    # rejected before any device pointer is touched
    st = f(limit + 1, 44, 1, 1, 1, 1, ctypes.byref(sel), None)
    assert st == gs.GS_ERR_CAPACITY
    assert b"exceed" in gs.lib.gs_stage_sort_noalloc_error()
