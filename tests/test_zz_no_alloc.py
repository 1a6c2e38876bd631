"""lgbm_b200_predict_noalloc (host buffers staged through the library's static
device array) against lgbm_b200_predict with host buffers, both through the C
ABI. Collected last so it also runs after every other test in one process."""
import ctypes as C
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(n, ncol, seed, nan_frac=0.05):
    r = np.random.default_rng(seed)
    X = r.standard_normal((n, ncol)).astype(np.float32)
    X[r.random((n, ncol)) < nan_frac] = np.nan
    return X


def _both(lgb, bst, X):
    L = lgb._lib
    k = bst.num_class
    want = np.full(X.shape[0] * k, np.nan, np.float64)
    L.check(L.lib().lgbm_b200_predict(bst._forest_handle(), X.ctypes.data, X.shape[0], X.shape[1],
                                      want.ctypes.data, L.HOST))
    got = []
    for _ in range(2):  # two calls in a row share the static array
        out = np.full(X.shape[0] * k, np.nan, np.float64)
        L.check(L.lib().lgbm_b200_predict_noalloc(bst._forest_handle(), X.ctypes.data, X.shape[0], X.shape[1],
                                                  out.ctypes.data))
        got.append(out)
    return want, got


def test_noalloc_binary_matches_predict(lgb):
    X = _rows(6000, 8, 1)
    y = (np.nan_to_num(X[:, 0]) + 0.5 * np.nan_to_num(X[:, 1]) > 0).astype(np.float32)
    bst = lgb.train({"objective": "binary", "num_leaves": 31}, lgb.Dataset(X, y), num_boost_round=15)
    want, got = _both(lgb, bst, _rows(5000, 8, 2))
    for g in got:
        assert np.array_equal(g, want)  # the same kernel on the same rows: bit-identical


def test_noalloc_multiclass_several_chunks(lgb):
    X = _rows(6000, 10, 3)
    y = (np.argmax(np.nan_to_num(X[:, :3]), axis=1)).astype(np.float32)
    bst = lgb.train({"objective": "multiclass", "num_class": 3, "num_leaves": 15}, lgb.Dataset(X, y),
                    num_boost_round=8)
    # 64 staging bytes per row: 262,140 rows per chunk, so 600,000 rows take three chunks
    Xt = _rows(600_000, 10, 4)
    want, got = _both(lgb, bst, Xt)
    for g in got:
        assert np.array_equal(g, want)
    # a smaller batch after the chunked one reuses the array
    X2 = _rows(3000, 10, 5)
    want2, got2 = _both(lgb, bst, X2)
    assert np.array_equal(got2[1], want2)


def test_noalloc_rejects_rows_above_the_staging_size(lgb):
    X = _rows(2000, 4, 6)
    y = (np.nan_to_num(X[:, 0]) > 0).astype(np.float32)
    bst = lgb.train({"objective": "binary", "num_leaves": 7}, lgb.Dataset(X, y), num_boost_round=2)
    L = lgb._lib
    tiny = np.zeros(4, np.float32)
    out = np.zeros(1, np.float64)
    ncol = (16 << 20) // 4  # one row alone needs 16 MiB + 8 bytes: rejected before any copy
    rc = L.lib().lgbm_b200_predict_noalloc(bst._forest_handle(), tiny.ctypes.data, 1, ncol, out.ctypes.data)
    assert rc == L.ERR_INVALID_PARAMETER
    assert b"16 MiB" in L.lib().lgbm_b200_last_error()
    # the entry point still works afterwards
    want, got = _both(lgb, bst, _rows(100, 4, 7))
    assert np.array_equal(got[0], want)


def test_noalloc_allocates_nothing_and_keeps_the_current_device(lgb):
    """The point of the entry point: a call on a forest the array has not
    served yet leaves the device's free memory unchanged, and the calling
    thread's current device is the same after the call. Two different
    forests use the shared array one after the other."""
    import torch

    X = _rows(6000, 8, 11)
    y = (np.nan_to_num(X[:, 0]) - np.nan_to_num(X[:, 2]) > 0).astype(np.float32)
    a = lgb.train({"objective": "binary", "num_leaves": 15}, lgb.Dataset(X, y), num_boost_round=6)
    b = lgb.train({"objective": "binary", "num_leaves": 31, "learning_rate": 0.3}, lgb.Dataset(X, y),
                  num_boost_round=9)
    L = lgb._lib
    Xt = _rows(20000, 8, 12)
    out = np.zeros(20000, np.float64)
    # warm-up with forest a: loads the kernel and resolves the array's address
    L.check(L.lib().lgbm_b200_predict_noalloc(a._forest_handle(), Xt.ctypes.data, 20000, 8, out.ctypes.data))
    hb = b._forest_handle()  # forest b's own arrays are allocated here, before the measurement
    torch.cuda.synchronize()
    before_dev = torch.cuda.current_device()
    gc.collect()  # no unrelated object may free device memory inside the window
    gc.disable()
    try:
        free0, _ = torch.cuda.mem_get_info()
        rc = L.lib().lgbm_b200_predict_noalloc(hb, Xt.ctypes.data, 20000, 8, out.ctypes.data)
        free1, _ = torch.cuda.mem_get_info()
    finally:
        gc.enable()
    L.check(rc)
    assert free1 == free0
    assert torch.cuda.current_device() == before_dev
    want_b, got_b = _both(lgb, b, Xt)
    assert np.array_equal(out, want_b)
    for g in got_b:
        assert np.array_equal(g, want_b)
    want_a, got_a = _both(lgb, a, Xt)  # back to forest a after b used the array
    assert np.array_equal(got_a[1], want_a)
