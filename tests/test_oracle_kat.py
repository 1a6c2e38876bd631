"""The oracle against the reference's own known-answer tests (the in-source
#[test]s of crates/lgbm-core). These are the oracle's parity pins."""
import ctypes as C
import math

import numpy as np
import pytest



def _oracle_binned(orc, lgb, x, params):
    """The oracle's own binning of x (binning.rs restated in oracle/binning.cpp)."""
    return orc.Dataset(x, lgb.resolve_params(params)).binned()


def _feature(orc, num_bin, missing_type, default_bin, mfb, bin_type, offset, penalty=1.0):
    return orc.OracleFeature(num_bin, missing_type, default_bin, mfb, bin_type, 0, offset, penalty, 0, 0.0, 0.0)


def _params(lgb, orc, **kw):
    # split.rs:1406-1421 test params
    base = dict(lambda_l1=0.0, lambda_l2=0.0, max_delta_step=0.0, path_smooth=0.0, min_data_in_leaf=1,
                min_sum_hessian_in_leaf=1e-3, min_gain_to_split=0.0, max_cat_to_onehot=4, max_cat_threshold=32,
                cat_l2=10.0, cat_smooth=10.0, min_data_per_group=100)
    base.update(kw)
    return orc.params_struct(lgb.resolve_params(base))


def _fbt(orc, f, ps, hist, sum_g, sum_h, n):
    out = orc.OracleSplit()
    h = np.ascontiguousarray(hist, dtype=np.float64)
    rc = orc.lib().oracle_find_best_threshold(C.byref(f), C.byref(ps), h.ctypes.data_as(C.POINTER(C.c_double)),
                                              None, sum_g, sum_h, 0, 0.0, 0.0, n, 0.0, C.byref(out))
    assert rc == 0
    return out


def test_finds_obvious_split(lgb, orc):  # split.rs:1423-1446
    f = _feature(orc, 4, 0, 0, 0, 0, 0)
    out = _fbt(orc, f, _params(lgb, orc), [-5.0, 5.0, -5.0, 5.0, 5.0, 5.0, 5.0, 5.0], 0.0, 20.0, 20)
    assert out.splittable
    assert out.threshold == 1
    assert out.left_count == 10
    assert abs(out.left_output - 1.0) < 1e-12
    assert abs(out.right_output + 1.0) < 1e-12
    assert abs(out.gain - 20.0) < 1e-9


def test_categorical_one_hot_and_sorted(lgb, orc):  # split.rs:1448-1474
    f = _feature(orc, 3, 2, 1, 1, 1, 0)
    out = _fbt(orc, f, _params(lgb, orc), [0.0, 10.0, -10.0, 10.0, 10.0, 10.0], 0.0, 30.0, 30)
    assert out.splittable
    assert list(out.cat_threshold[: out.num_cat]) == [1]
    assert not out.default_left
    assert out.left_count == 10
    f = _feature(orc, 6, 2, 0, 0, 1, 1)
    hist = [5.0, 100.0, -50.0, 100.0, 2.0, 100.0, -40.0, 100.0, 3.0, 100.0]
    out = _fbt(orc, f, _params(lgb, orc, min_data_per_group=1, cat_smooth=1.0), hist, -80.0, 600.0, 600)
    assert out.splittable
    assert sorted(out.cat_threshold[: out.num_cat]) == [2, 4]


def test_l1_and_max_delta_step(lgb, orc):  # split.rs:1486-1493 via a one-bin-per-side split
    # leaf_output(-10, 2) with l1 = 1, max_delta_step = 0.5 clamps to 0.5
    f = _feature(orc, 2, 0, 0, 0, 0, 0)
    ps = _params(lgb, orc, lambda_l1=1.0, max_delta_step=0.5)
    out = _fbt(orc, f, ps, [-10.0, 2.0, 10.0, 2.0], 0.0, 4.0, 20)
    assert out.left_output == 0.5
    assert out.right_output == -0.5


def test_to_i8_casts_like_x86(orc):  # quant.rs:484-491
    L = orc.lib()
    assert L.oracle_to_i8(2.7) == 2
    assert L.oracle_to_i8(-2.7) == -2
    assert L.oracle_to_i8(200.0) == -56
    assert L.oracle_to_i8(float("nan")) == 0
    assert L.oracle_to_i8(1e300) == 0


def test_quant_packing(orc):  # quant.rs:493-503
    g = np.array([1.0, -0.5], np.float32)
    h = np.array([0.5, 0.25], np.float32)
    packed = np.zeros(2, np.int64)
    scales = np.zeros(2, np.float64)
    rc = orc.lib().oracle_discretize(4, 0, 0, 0, 2, 1, 1, g.ctypes.data_as(C.POINTER(C.c_float)),
                                     h.ctypes.data_as(C.POINTER(C.c_float)),
                                     packed.ctypes.data_as(C.POINTER(C.c_int64)),
                                     scales.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    assert list(scales) == [0.5, 0.125]
    assert packed[1] == (-1 << 32) | 2
    assert packed[0] == (2 << 32) | 4
    assert (packed[0] + packed[1]) == (1 << 32) | 6


def test_block_info(orc):  # multi_val_bin.rs:832-838
    out = np.zeros(2, np.int64)
    for args, want in [((1, 1000, 77), (1, 1000)), ((16, 1000, 77), (13, 96)), ((16, 1000000, 77), (16, 62528)),
                       ((4, 50, 77), (1, 50))]:
        orc.lib().oracle_block_info(*args, out.ctypes.data_as(C.POINTER(C.c_int64)))
        assert tuple(out) == want


def test_mt19937_standard_sequence(orc):  # mt19937.rs:200-209
    out = np.zeros(10000, np.uint32)
    orc.lib().oracle_mt19937(5489, 10000, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert out[-1] == 4123659995


def test_lcg_sample(orc):  # random.rs:77-105
    out = np.zeros(1000, np.int32)
    n = C.c_int32()
    orc.lib().oracle_lcg_sample(1, 5, 5, out.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n))
    assert list(out[: n.value]) == [0, 1, 2, 3, 4]
    for nn, k in [(1000, 10), (1000, 900), (50000, 20000)]:
        buf = np.zeros(k, np.int32)
        orc.lib().oracle_lcg_sample(7, nn, k, buf.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n))
        s = buf[: n.value]
        assert np.all(np.diff(s) > 0)
        if k <= 10:
            assert n.value == k
        assert s.min() >= 0 and s.max() < nn


def test_auc_perfect_and_ties(orc):  # metric.rs:866-871
    assert orc.auc(np.array([0, 0, 1, 1.0]), np.array([0.1, 0.2, 0.8, 0.9])) == 1.0
    assert orc.auc(np.array([0, 0, 1, 1.0]), np.array([0.5, 0.5, 0.5, 0.5])) == 0.5


def test_ndcg_values(orc):  # metric.rs:910-918 (eval_at 2,1 reported as @1, @2)
    v = orc.ndcg(np.array([0.0, 1.0, 0.0, 0.0]), np.array([1.0, 0.0, 0.0, 0.0]), [2, 2], [1, 2])
    assert list(v) == [(0.0 + 1.0) / 2.0, (1.0 / math.log2(3.0) + 1.0) / 2.0]


def test_lambdarank_pair_gradients(lgb, orc):  # rank.rs:492-510
    p = lgb.resolve_params({"objective": "lambdarank", "lambdarank_norm": False})
    g, h = orc.gradients(p, np.array([1.0, 0.0]), np.array([0.0, 0.0]), group=[2])
    dndcg = 1.0 * (1.0 - 1.0 / math.log2(3.0))
    # get_sigmoid(0) reads the table entry at (0 - min) * factor
    idx = int((0.0 + 25.0) * (1024 * 1024 / 50.0))
    p0 = 1.0 / (1.0 + math.exp((idx / (1024 * 1024 / 50.0) - 25.0) * 1.0))
    assert abs(p0 - 0.5) < 1e-4
    lam = np.float32(p0 * -dndcg)
    assert list(g) == [lam, -lam]
    hh = np.float32(p0 * (1.0 - p0) * dndcg)
    assert list(h) == [hh, hh]


def _step_data(n):  # learner/tests.rs:6-17
    x = np.zeros((n, 2), np.float64)
    y = np.zeros(n, np.float32)
    for i in range(n):
        a = i / n
        x[i] = (a, float((i * 37) % 11))
        y[i] = -1.0 if a < 0.5 else 1.0
    return x, y


def test_first_split_separates_step(lgb, orc):  # learner/tests.rs:24-43
    n = 200
    x, y = _step_data(n)
    params = {"num_leaves": 2, "min_data_in_leaf": 5}
    b = _oracle_binned(orc, lgb, x.astype(np.float32), params)
    grad = -y
    hess = np.ones(n, np.float32)
    t = orc_tree(lgb, orc, b, params, grad, hess)
    assert t["num_leaves"] == 2
    assert t["split_feature"][0] == 0
    assert list(t["leaf_count"]) == [100, 100]
    assert abs(t["leaf_value"][0] + 1.0) < 1e-9
    assert abs(t["leaf_value"][1] - 1.0) < 1e-9


def test_max_depth_and_min_data(lgb, orc):  # learner/tests.rs:64-78
    n = 300
    x, y = _step_data(n)
    params = {"num_leaves": 31, "max_depth": 2, "min_data_in_leaf": 40}
    b = _oracle_binned(orc, lgb, x.astype(np.float32), params)
    grad = np.sin(np.arange(n, dtype=np.float32) * np.float32(0.37)).astype(np.float32)
    t = orc_tree(lgb, orc, b, params, grad, np.ones(n, np.float32))
    assert t["num_leaves"] <= 4
    assert t["leaf_depth"].max() <= 2
    assert all(c >= 40 for c in t["leaf_count"])


def test_constant_gradient_single_leaf(lgb, orc):  # learner/tests.rs:80-89
    n = 100
    x, y = _step_data(n)
    b = _oracle_binned(orc, lgb, x.astype(np.float32), {})
    t = orc_tree(lgb, orc, b, {}, np.full(n, 0.5, np.float32), np.ones(n, np.float32))
    assert t["num_leaves"] == 1


def orc_tree(lgb, orc, b, params, grad, hess):
    """One tree of the oracle learner on given gradients (a custom-objective iteration)."""
    return orc.train_trees(lgb.resolve_params(params), b, grad, hess).trees[0]


def test_fix_recovers_most_frequent_bin(orc):  # histogram.rs:91-97
    # bins 0,1,1,2 with gradients 1,2,3,4 and mfb = 1: bin 1 is not stored
    hist = np.array([1.0, 1.0, 0.0, 0.0, 4.0, 1.0])
    assert orc.lib().oracle_fix_hist(3, 0, 1, 10.0, 4.0, hist.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert list(hist) == [1.0, 1.0, 5.0, 2.0, 4.0, 1.0]


def test_offset_one_leaves_the_histogram_alone(orc):  # histogram.rs:99-106
    hist = np.array([2.0, 1.0, 3.0, 1.0])  # 2 * (num_bin - offset) values
    assert orc.lib().oracle_fix_hist(3, 1, 0, 7.0, 3.0, hist.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert list(hist) == [2.0, 1.0, 3.0, 1.0]


def test_tie_break_prefers_smaller_feature(orc):  # split.rs:1476-1484
    L = orc.lib()
    assert L.oracle_better_than(1.0, 1, 1.0, 3) == 1  # b (feature 1) beats a (feature 3) at equal gain
    assert L.oracle_better_than(1.0, 3, 1.0, 1) == 0
    assert L.oracle_better_than(1.0, 3, -math.inf, -1) == 1  # any split beats the default (none)


def test_partition_is_stable(lgb, orc):  # learner/tests.rs:45-63
    n = 100
    x, y = _step_data(n)
    params = {"num_leaves": 4, "min_data_in_leaf": 3}
    b = _oracle_binned(orc, lgb, x.astype(np.float32), params)
    grad = np.array([((i * 7919) % 13) - 6.0 for i in range(n)], np.float32)
    m = orc.train_trees(lgb.resolve_params(params), b, grad, np.ones(n, np.float32))
    t = m.trees[0]
    beg, cnt, idx = orc.partition(m, t["num_leaves"], n)
    seen = 0
    for leaf in range(t["num_leaves"]):
        rows = idx[beg[leaf]: beg[leaf] + cnt[leaf]].astype(np.int64)
        assert np.all(np.diff(rows) > 0), f"leaf {leaf} indices not increasing"
        seen += len(rows)
    assert seen == n


def bin_rs_histogram_case():
    """bin.rs:762-788: 300 rows, stored value 1 + i % 3 on every 7th row and
    0 (the most frequent bin, not stored) elsewhere; gradients and hessians
    i * 0.5; the rows with i % 3 != 1. Returns (binned, g, rows, want): a
    one-feature binned dataset holding those stored values (num_bin 4, most
    frequent bin 0) and the (g, h) sums of stored values 1..3."""
    n = 300
    vals = np.array([(1 + i % 3) if i % 7 == 0 else 0 for i in range(n)], np.uint8)
    g = (np.arange(n, dtype=np.float32) * np.float32(0.5)).astype(np.float32)
    rows = np.array([i for i in range(n) if i % 3 != 1], np.uint32)
    want = np.zeros(8)
    for i in rows:
        v = int(vals[i])
        if v != 0:
            want[2 * v] += float(g[i])
            want[2 * v + 1] += float(g[i])
    b = {"num_data": n, "num_features": 1, "num_total_features": 1, "bins": vals.reshape(n, 1),
         "num_bin": np.array([4], np.int32), "missing_type": np.array([0], np.int32),
         "default_bin": np.array([0], np.int32), "most_freq_bin": np.array([0], np.int32),
         "bin_type": np.array([0], np.int32), "real_index": np.array([0], np.int32),
         "upper_bounds": np.array([1e-35, 1.5, 2.5, np.inf]), "ub_offsets": np.array([0, 4], np.int64),
         "bin_to_cat": np.zeros(0, np.int32), "cat_offsets": np.array([0, 0], np.int64)}
    return b, g, rows, want[2:]


def test_bin_histogram_matches_dense_reference(orc):  # bin.rs:762-788 (the histogram part)
    b, g, rows, want = bin_rs_histogram_case()
    got = orc.hist(b, rows, g, g)
    assert list(got) == list(want)
