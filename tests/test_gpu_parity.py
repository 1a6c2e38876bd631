"""Parity of the CUDA tree-learning path with the CPU oracle, through the C ABI.

Tolerances:
  - bins, per-bin integer sums, leaf row sets, tree structure: exact;
  - FP64 histogram sums: 1e-12 relative to the oracle's single-threaded
    row-order sums (atomics reorder the additions);
  - split gains / leaf values: 1e-10 / 1e-9 relative;
  - quantized form: integer histograms and trees exact.
"""
import numpy as np
import pytest

from conftest import TOL, binned_dataset, compare_boosted_trees, within

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["per_step", "persistent", "scan_part"])
def grow_mode(request, lgb, monkeypatch):
    """Every test runs with each launch strategy: the per-step graph (the
    default), persistent growth, and the scans and the partition of a step
    in one cooperative launch."""
    from lgbm_b200 import basic

    monkeypatch.setitem(basic.DEFAULTS, "persistent_grow", request.param == "persistent")
    monkeypatch.setenv("LGBM_B200_SCANPART", "1" if request.param == "scan_part" else "0")
    yield request.param


def _binary_data(n, f=28, seed=0, nan_frac=0.0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    z = X[:, 0] + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2 + 0.3 * rng.standard_normal(n)
    y = (rng.random(n) < 1 / (1 + np.exp(-z))).astype(np.float32)
    if nan_frac:
        X[rng.random(X.shape) < nan_frac] = np.nan
    return X, y


# Gain ties the device resolves differently from the oracle, by (tree, node):
# two candidates whose FP64 gains agree within the [split_gain] tie_rtol. A
# divergence not listed here fails its test.
DOCUMENTED_TIES = {"binary_30_rounds": set(), "lambdarank_8_rounds": set()}


def _grads(orc, p, y, scores=None):
    if scores is None:
        scores = np.zeros(len(y))
    return orc.gradients(p, y, scores)


def assert_same_tree(a, b, leaf_rtol=None, gain_rtol=None, gains=None):
    """Structure exact; leaf values within leaf_rtol (tests/tolerances.toml
    [leaf_value] by default); the FP64 split gains within gain_rtol
    ([split_gain]) of the oracle's trace `gains`, and the stored f32 gains
    within one f32 ulp (an FP64 gain within 1e-10 can round either way)."""
    leaf_rtol = TOL["leaf_value"]["rtol"] if leaf_rtol is None else leaf_rtol
    gain_rtol = TOL["split_gain"]["rtol"] if gain_rtol is None else gain_rtol
    assert a["num_leaves"] == b["num_leaves"], (a["num_leaves"], b["num_leaves"])
    for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child", "leaf_count",
              "internal_count", "leaf_depth"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    for k in ("leaf_value", "leaf_weight", "internal_value", "internal_weight"):
        np.testing.assert_allclose(a[k], b[k], rtol=leaf_rtol, atol=TOL["leaf_value"]["atol"], err_msg=k)
    if gains is not None:
        np.testing.assert_allclose(a["split_gain_f64"], gains, rtol=gain_rtol, atol=0.0, err_msg="split_gain_f64")
    ulps = np.abs(np.asarray(a["split_gain"], np.float32).view(np.int32).astype(np.int64) -
                  np.asarray(b["split_gain"], np.float32).view(np.int32).astype(np.int64))
    assert ulps.max(initial=0) <= (0 if gain_rtol == 0.0 else 1), "split_gain (f32)"


@pytest.mark.parametrize("form", ["f64", "f32c"])
def test_histogram_float_forms(lgb, orc, form):
    X, y = _binary_data(60000, seed=1, nan_frac=0.02)
    params = {"objective": "binary", "hist_precision": form}
    ds = binned_dataset(lgb, X, y, params)
    b = ds.binned()
    p = lgb.resolve_params(params)
    g, h = _grads(orc, p, y, np.random.default_rng(2).standard_normal(len(y)) * 0.5)
    learner = lgb.Learner(ds, params)
    learner.train(g, h)  # loads the gradients into the learner
    rng = np.random.default_rng(3)
    for rows in (None, np.sort(rng.choice(len(y), 20000, replace=False)).astype(np.uint32),
                 np.sort(rng.choice(len(y), 37, replace=False)).astype(np.uint32)):
        got = learner.histogram(rows)
        want = orc.hist(b, rows, g, h)
        scale = np.maximum(np.abs(want), 1e-300)
        err = np.max(np.abs(got - want) / np.maximum(scale, np.abs(want).max() * 1e-16 + 1e-300))
        tol = 1e-12 if form == "f64" else 1e-7
        assert err < tol, (form, err)


def test_quantized_gradients_and_histogram_exact(lgb, orc):
    X, y = _binary_data(50000, seed=4)
    params = {"objective": "binary", "use_quantized_grad": True, "num_grad_quant_bins": 4, "num_threads": 8,
              "seed": 7}
    ds = binned_dataset(lgb, X, y, params)
    b = ds.binned()
    p = lgb.resolve_params(params)
    g, h = _grads(orc, p, y, np.random.default_rng(5).standard_normal(len(y)))
    learner = lgb.Learner(ds, params)
    learner.train(g, h)
    packed, scales = learner.quantized()
    # the oracle's discretizer after one call with the same seed / thread count
    import ctypes as C

    want = np.zeros(len(y), np.int64)
    ws = np.zeros(2)
    orc.lib().oracle_discretize(4, int(p["seed"]), 0, 1, len(y), 8, 1,
                                g.ctypes.data_as(C.POINTER(C.c_float)), h.ctypes.data_as(C.POINTER(C.c_float)),
                                want.ctypes.data_as(C.POINTER(C.c_int64)), ws.ctypes.data_as(C.POINTER(C.c_double)))
    assert list(scales) == list(ws)
    assert np.array_equal(packed, want)
    rows = np.sort(np.random.default_rng(6).choice(len(y), 12345, replace=False)).astype(np.uint32)
    got = learner.histogram(rows)
    total = int(np.sum(b["num_bin"] - (b["most_freq_bin"] == 0)))
    exp = np.zeros(total, np.int64)
    d = orc.Data(b)
    orc.lib().oracle_hist(C.byref(d.s), rows.ctypes.data_as(C.POINTER(C.c_uint32)), len(rows), None, None,
                          want.ctypes.data_as(C.POINTER(C.c_int64)), None, exp.ctypes.data_as(C.POINTER(C.c_int64)))
    assert np.array_equal(got, exp)


def _tree_pair(lgb, orc, X, y, params, grad_scores=None, categorical=None, bag=None, mask=None):
    ds = binned_dataset(lgb, X, y, params, categorical=categorical)
    b = ds.binned()
    p = lgb.resolve_params(params)
    g, h = _grads(orc, p, y, grad_scores)
    learner = lgb.Learner(ds, params)
    if bag is not None:
        learner.set_bagging(bag)
    if mask is not None:
        learner.set_feature_mask(0, mask)
    gt = learner.train(g, h)[0]
    om = orc.train_trees(p, b, g, h, bag=bag, bytree=None if mask is None else mask.reshape(1, -1))
    return gt, om.trees[0], learner, om, b


@pytest.mark.parametrize("num_leaves", [2, 31, 255])
def test_single_tree_f64(lgb, orc, num_leaves):
    X, y = _binary_data(20000, seed=10)
    params = {"objective": "binary", "num_leaves": num_leaves, "min_data_in_leaf": 20}
    gt, ot, learner, om, b = _tree_pair(lgb, orc, X, y, params)
    assert_same_tree(gt, ot, gains=om.trace(0)[3])
    # leaf row lists are exact, in the reference's (ascending) order
    beg, cnt, idx = learner.partition(0, gt["num_leaves"])
    obeg, ocnt, oidx = orc.partition(om, ot["num_leaves"], len(y))
    for leaf in range(gt["num_leaves"]):
        a = idx[beg[leaf]: beg[leaf] + cnt[leaf]]
        o = oidx[obeg[leaf]: obeg[leaf] + ocnt[leaf]]
        assert np.array_equal(a, o), leaf


def test_single_tree_nan_missing_and_regularisation(lgb, orc):
    X, y = _binary_data(30000, seed=11, nan_frac=0.05)
    params = {"objective": "binary", "num_leaves": 63, "min_data_in_leaf": 10, "lambda_l1": 0.5,
              "lambda_l2": 2.0, "max_delta_step": 0.7, "min_gain_to_split": 0.01}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, y, params)
    assert_same_tree(gt, ot, gains=om.trace(0)[3])


def test_single_tree_path_smooth_and_depth(lgb, orc):
    X, y = _binary_data(20000, seed=12)
    params = {"objective": "binary", "num_leaves": 63, "max_depth": 5, "path_smooth": 3.0}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, y, params)
    assert_same_tree(gt, ot, gains=om.trace(0)[3])


def test_single_tree_categorical(lgb, orc):
    rng = np.random.default_rng(13)
    n = 30000
    X = rng.standard_normal((n, 6)).astype(np.float32)
    p = 1.0 / np.arange(1, 31) ** 1.2
    p /= p.sum()
    X[:, 4] = rng.choice(30, n, p=p)
    X[:, 5] = rng.integers(0, 3, n)
    eff = rng.standard_normal(30)
    y = (X[:, 0] + eff[X[:, 4].astype(int)] + 0.5 * (X[:, 5] == 1) + 0.3 * rng.standard_normal(n) > 0)
    params = {"objective": "binary", "num_leaves": 31, "max_cat_to_onehot": 4, "min_data_per_group": 50,
              "cat_smooth": 5.0}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, y.astype(np.float32), params, categorical=[4, 5])
    assert gt["num_cat"] > 0
    assert_same_tree(gt, ot, gains=om.trace(0)[3])
    assert np.array_equal(gt["cat_boundaries"], ot["cat_boundaries"])
    assert np.array_equal(gt["cat_threshold"], ot["cat_threshold"])


def test_single_tree_bagging_and_feature_mask(lgb, orc):
    X, y = _binary_data(25000, seed=14, nan_frac=0.03)
    rng = np.random.default_rng(15)
    bag = np.sort(rng.choice(len(y), 18000, replace=False)).astype(np.uint32)
    mask = (rng.random(X.shape[1]) < 0.7).astype(np.uint8)
    params = {"objective": "regression", "num_leaves": 127}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, rng.standard_normal(len(y)).astype(np.float32), params, bag=bag,
                                  mask=mask)
    assert_same_tree(gt, ot, gains=om.trace(0)[3])
    assert set(gt["split_feature"]) <= set(np.nonzero(mask)[0])


def test_single_tree_monotone(lgb, orc):
    X, y = _binary_data(20000, seed=16)
    mono = [1, -1, 0, 0] + [0] * 24
    params = {"objective": "binary", "num_leaves": 31, "monotone_constraints": mono, "monotone_penalty": 0.5}
    ds = binned_dataset(lgb, X, y, params)
    b = ds.binned()
    p = lgb.resolve_params(params)
    g, h = orc.gradients(p, y, np.zeros(len(y)))
    learner = lgb.Learner(ds, params)
    gt = learner.train(g, h)[0]
    om = orc.train_trees(p, b, g, h, monotone=mono)
    assert_same_tree(gt, om.trees[0], gains=om.trace(0)[3])


@pytest.mark.parametrize("renew", [False, True])
def test_single_tree_quantized_exact(lgb, orc, renew):
    X, y = _binary_data(40000, seed=17)
    params = {"objective": "binary", "num_leaves": 127, "use_quantized_grad": True, "num_threads": 16,
              "quant_train_renew_leaf": renew}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, y, params)
    gains = om.trace(0)[3]
    if renew:  # leaf outputs re-fit from FP64 gradient sums (summation order differs)
        assert_same_tree(gt, ot, leaf_rtol=1e-12, gain_rtol=0.0, gains=gains)
    else:
        assert_same_tree(gt, ot, leaf_rtol=0.0, gain_rtol=0.0, gains=gains)


@pytest.mark.parametrize("per", [1, 8])
def test_single_tree_quantized_warp_scan(lgb, orc, grow_mode, monkeypatch, per):
    """The quantized scan by one warp per (feature, side), forced on a step of
    few items (by default it runs only when the block scans would take several
    waves): NaN missing values in both scan directions, L1/L2, max_delta_step
    and two categorical features (one-hot and sorted). Integer sums make it
    bit-exact with the oracle, as the block scan is; `per` items share a CTA."""
    if grow_mode != "per_step":
        pytest.skip("the warp scan is a launch of the per-step graph")
    monkeypatch.setenv("LGBM_B200_SCAN_WARP", "1")
    monkeypatch.setenv("LGBM_B200_SCAN_PER", str(per))
    rng = np.random.default_rng(21)
    X, y = _binary_data(30000, f=12, seed=21, nan_frac=0.05)
    pz = 1.0 / np.arange(1, 41) ** 1.1
    X[:, 10] = rng.choice(40, len(y), p=pz / pz.sum())
    X[:, 11] = rng.integers(0, 3, len(y))
    params = {"objective": "binary", "num_leaves": 63, "use_quantized_grad": True, "num_threads": 16,
              "lambda_l1": 0.3, "lambda_l2": 1.5, "max_delta_step": 0.8, "max_cat_to_onehot": 4,
              "min_data_per_group": 50, "cat_smooth": 5.0}
    gt, ot, _, om, _ = _tree_pair(lgb, orc, X, y, params, categorical=[10, 11])
    assert_same_tree(gt, ot, leaf_rtol=0.0, gain_rtol=0.0, gains=om.trace(0)[3])
    assert np.array_equal(gt["cat_boundaries"], ot["cat_boundaries"])
    assert np.array_equal(gt["cat_threshold"], ot["cat_threshold"])


def test_multiclass_slots_in_lockstep(lgb, orc):
    rng = np.random.default_rng(18)
    n = 15000
    X = rng.standard_normal((n, 10)).astype(np.float32)
    y = np.argmax(X[:, :3] + 0.5 * rng.standard_normal((n, 3)), axis=1).astype(np.float32)
    params = {"objective": "multiclass", "num_class": 3, "num_leaves": 31}
    ds = binned_dataset(lgb, X, y, params)
    b = ds.binned()
    p = lgb.resolve_params(params)
    scores = rng.standard_normal(3 * n) * 0.3
    g, h = orc.gradients(p, y, scores)
    learner = lgb.Learner(ds, params, num_tree_slots=3)
    gts = learner.train(g, h)
    om = orc.train_trees(p, b, g, h, num_trees=3)
    for k in range(3):
        assert_same_tree(gts[k], om.trees[k], gains=om.trace(k)[3])


def test_gradients(lgb, orc):
    rng = np.random.default_rng(19)
    n = 100000
    s = rng.standard_normal(n) * 3
    yb = (rng.random(n) < 0.4).astype(np.float32)
    for params, y, sc in (({"objective": "binary"}, yb, s), ({"objective": "regression"}, rng.standard_normal(n), s),
                          ({"objective": "multiclass", "num_class": 4}, rng.integers(0, 4, n).astype(np.float32),
                           rng.standard_normal(4 * n))):
        p = lgb.resolve_params(params)
        g, h = lgb.gradients(params, y, sc)
        og, oh = orc.gradients(p, y, sc)
        # exp is not correctly rounded on either side: allow one f32 ulp
        for a, o in ((g, og), (h, oh)):
            ulps = np.abs(a.view(np.int32).astype(np.int64) - o.view(np.int32).astype(np.int64))
            assert ulps.max() <= 1, (params, ulps.max())
            assert np.mean(ulps == 0) > 0.99


def test_boosting_matches_oracle(lgb, orc):
    """30 rounds: every tree as the oracle's (structure exact, gains and leaf
    values within tests/tolerances.toml) unless the device meets a gain tie,
    which must be a tie within [split_gain] tie_rtol; with no tie the held-out
    scores and AUC agree within the [predictions] / [metrics] bars."""
    X, y = _binary_data(12000, seed=20)
    Xv, yv = _binary_data(3000, seed=21)
    params = {"objective": "binary", "num_leaves": 31, "learning_rate": 0.1, "min_data_in_leaf": 20}
    rounds = 30
    ds = lgb.Dataset(X, y, params=params)
    dv = lgb.Dataset(Xv, yv, params=params, reference=ds)
    bst = lgb.train(params, ds, rounds, valid_sets=[dv])
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, rounds, valid_binned=dv.binned())
    assert bst.num_trees() == len(om.trees)
    same, tie = compare_boosted_trees(bst.trees, om)
    assert tie is None or tie[:2] in DOCUMENTED_TIES["binary_30_rounds"], tie
    if tie is None:
        assert same == rounds
        assert within(bst.scores(valid=True)[0], om.scores(valid=True)[0], "predictions")
        assert within(orc.auc(yv, bst.scores(valid=True)[0]), orc.auc(yv, om.scores(valid=True)[0]), "metrics")
    # batched prediction of the GPU model on raw features equals its binned valid scores
    raw = bst.predict(Xv, raw_score=True)
    assert within(raw, bst.scores(valid=True)[0], "predictions")


def test_predict_matches_oracle(lgb, orc):
    X, y = _binary_data(8000, seed=22, nan_frac=0.05)
    params = {"objective": "binary", "num_leaves": 15}
    ds = lgb.Dataset(X, y, params=params)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, 20)
    bst = lgb.Booster(params)
    bst.trees = [dict(t, leaf_parent=np.zeros(t["num_leaves"], np.int32),
                      cat_boundaries_inner=np.zeros(1, np.int32), cat_threshold_inner=np.zeros(0, np.uint32))
                 for t in om.trees]
    Xt, _ = _binary_data(5000, seed=23, nan_frac=0.05)
    got = bst.predict(Xt, raw_score=True)
    want = om.predict_raw(Xt)[:, 0]
    assert np.array_equal(got, want)


def _ranking_data(nq, f=16, seed=0):
    rng = np.random.default_rng(seed)
    group = np.clip(rng.geometric(1 / 20, nq), 1, 200).astype(np.int32)
    n = int(group.sum())
    X = rng.standard_normal((n, f)).astype(np.float32)
    X[rng.random(X.shape) < 0.2] = 0.0
    s = X[:, 0] + 0.5 * X[:, 1] - 0.3 * X[:, 2] * X[:, 3] + 0.5 * rng.standard_normal(n)
    y = np.digitize(s, np.quantile(s, [0.5, 0.75, 0.9, 0.97])).astype(np.float32)
    return X, y, group


def test_lambdarank_boosting_matches_oracle(lgb, orc):
    """8 lambdarank rounds: trees as the oracle's up to a documented gain tie,
    NDCG@1/3/5/10 of the scores within the [metrics] bar when no tie."""
    X, y, group = _ranking_data(400, seed=30)
    params = {"objective": "lambdarank", "num_leaves": 31, "min_data_in_leaf": 20, "learning_rate": 0.1}
    rounds = 8
    ds = lgb.Dataset(X, y, group=group, params=params)
    bst = lgb.train(params, ds, rounds)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, rounds, group=group)
    assert bst.num_trees() == len(om.trees)
    same, tie = compare_boosted_trees(bst.trees, om)
    assert tie is None or tie[:2] in DOCUMENTED_TIES["lambdarank_8_rounds"], tie
    if tie is None:
        assert same == rounds
        ks = [1, 3, 5, 10]
        got = orc.ndcg(y, bst.scores()[0], group, ks)
        want = orc.ndcg(y, om.scores()[0], group, ks)
        assert within(got, want, "metrics"), (got, want)


def _multiclass_categorical(n, seed):
    """The multiclass K=10 workload's generator (180 N(0,1) + 20 categorical
    features, Zipf s=1.2 over 50 categories), reduced to n rows."""
    from lgbm_b200 import synthetic

    d = synthetic.config3(scale=n / 2_000_000, seed=seed)
    return d["X"], d["y"], d["categorical"]


@pytest.mark.parametrize("renew", [False, True])
def test_quantized_categorical_multiclass_matches_oracle(lgb, orc, renew, grow_mode):
    """Config 3's form (quantized, K=10 trees per iteration, 20 Zipf
    categorical features, max_cat_to_onehot 4) on 50k rows: three boosting
    iterations. The integer histograms and the integer categorical scan
    (split.rs:1190-1400) make every tree bit-exact with the oracle; with
    FP64 leaf renewal the leaf values follow the leaf_value bar."""
    from conftest import TOL

    if grow_mode != "per_step":
        pytest.skip("the booster runs the default launch strategy")
    X, y, cats = _multiclass_categorical(50_000, seed=8)
    params = {"objective": "multiclass", "num_class": 10, "num_leaves": 127, "max_cat_to_onehot": 4,
              "use_quantized_grad": True, "num_grad_quant_bins": 4, "num_threads": 16, "seed": 11,
              "quant_train_renew_leaf": renew}
    ds = lgb.Dataset(X, y, params=params, categorical_feature=cats)
    bst = lgb.train(params, ds, 3)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, 3)
    assert bst.num_trees() == len(om.trees) == 30
    assert sum(t["num_cat"] for t in om.trees) > 0  # categorical splits are taken
    for i, (a, o) in enumerate(zip(bst.trees, om.trees)):
        for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child",
                  "leaf_count", "cat_boundaries", "cat_threshold"):
            assert np.array_equal(np.asarray(a[k]), np.asarray(o[k])), (i, k)
        if renew:
            tol = TOL["leaf_value"]
            np.testing.assert_allclose(a["leaf_value"], o["leaf_value"], rtol=tol["rtol"], atol=tol["atol"])
        else:
            assert np.array_equal(a["leaf_value"], o["leaf_value"]), i
            assert np.array_equal(a["split_gain"], o["split_gain"]), i
