"""Launch shapes of the per-step kernels (lgbm_b200_learner_set_launch_shape)
and the autotuner's measurement (lgbm_b200_learner_autotune).

No shape changes a result: learners that differ only in their launch shape
grow the same trees from the same gradients (quantized form: exactly; FP64
form: the same splits and row sets, values within the FP64 bars, since the
histogram atomics add in another order). The autotuner regrows the last
tree and leaves the random streams of later trees untouched."""
import numpy as np
import pytest

from conftest import binned_dataset

pytestmark = pytest.mark.gpu

SHAPES = [
    {"partition_ctas": 1, "hist_ctas": 8, "hist_rows_per_block": 32},
    {"partition_ctas": 7, "hist_ctas": 24, "hist_rows_per_block": 4096},
    {"partition_ctas": 2000, "hist_ctas": 600, "hist_rows_per_block": 300},
]


def _data(n, f=20, seed=0, classes=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    X[rng.random(X.shape) < 0.02] = np.nan
    z = np.nan_to_num(X[:, 0] + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2) + 0.3 * rng.standard_normal(n)
    if classes:
        y = np.digitize(z, np.quantile(z, np.linspace(0, 1, classes + 1)[1:-1])).astype(np.float32)
    else:
        y = (rng.random(n) < 1 / (1 + np.exp(-z))).astype(np.float32)
    return X, y


def _params(form, classes=0):
    p = {"objective": "multiclass" if classes else "binary", "num_leaves": 63, "min_data_in_leaf": 20,
         "num_threads": 8, "seed": 11}
    if classes:
        p["num_class"] = classes
    if form == "quantized":
        p.update(use_quantized_grad=True, num_grad_quant_bins=4, stochastic_rounding=True)
    else:
        p["hist_precision"] = form
    return p


def _grads(lgb, params, y, k, seed):
    s = np.random.default_rng(seed).standard_normal(k * len(y))
    return lgb.gradients(params, y, s)


def _same(a, b, exact):
    assert a["num_leaves"] == b["num_leaves"]
    for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child", "leaf_count",
              "internal_count"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    for k in ("leaf_value", "internal_value", "split_gain"):
        if exact:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
        else:
            np.testing.assert_allclose(a[k], b[k], rtol=1e-9, atol=1e-12, err_msg=k)


def _leaf_sets(learner, slot, nl):
    beg, cnt, idx = learner.partition(slot, nl)
    return [np.sort(idx[beg[i]:beg[i] + cnt[i]]) for i in range(nl)]


@pytest.mark.parametrize("form,scan_part", [("quantized", "0"), ("quantized", "1"), ("f64", "0")])
@pytest.mark.parametrize("shape", range(len(SHAPES)))
def test_shape_grows_the_same_trees(lgb, monkeypatch, form, scan_part, shape):
    monkeypatch.setenv("LGBM_B200_SCANPART", scan_part)
    X, y = _data(120_000, seed=1)
    params = _params(form)
    ds = binned_dataset(lgb, X, y, params)
    base = lgb.Learner(ds, params)
    other = lgb.Learner(ds, params)
    other.launch_shape = SHAPES[shape]
    got = other.launch_shape
    assert got["partition_ctas"] == SHAPES[shape]["partition_ctas"]
    assert got["hist_rows_per_block"] == SHAPES[shape]["hist_rows_per_block"]
    assert SHAPES[shape]["hist_ctas"] <= got["hist_ctas"] < SHAPES[shape]["hist_ctas"] + 16  # whole clusters
    for it in range(2):  # the second tree draws the next quantization offset
        g, h = _grads(lgb, params, y, 1, 100 + it)
        a = base.train(g, h)[0]
        b = other.train(g, h)[0]
        _same(a, b, exact=form == "quantized")
        nl = int(a["num_leaves"])
        for ra, rb in zip(_leaf_sets(base, 0, nl), _leaf_sets(other, 0, nl)):
            assert np.array_equal(ra, rb)


def test_shape_multiclass_slots(lgb):
    X, y = _data(60_000, seed=2, classes=3)
    params = _params("quantized", classes=3)
    ds = binned_dataset(lgb, X, y, params)
    base = lgb.Learner(ds, params, num_tree_slots=3)
    other = lgb.Learner(ds, params, num_tree_slots=3)
    other.launch_shape = {"partition_ctas": 12, "hist_ctas": 16, "hist_rows_per_block": 128}
    g, h = _grads(lgb, params, y, 3, 7)
    for a, b in zip(base.train(g, h), other.train(g, h)):
        _same(a, b, exact=True)


def test_autotune_regrows_and_keeps_streams(lgb):
    X, y = _data(120_000, seed=3)
    params = _params("quantized")
    ds = binned_dataset(lgb, X, y, params)
    tuned = lgb.Learner(ds, params)
    plain = lgb.Learner(ds, params)
    g1, h1 = _grads(lgb, params, y, 1, 1)
    g2, h2 = _grads(lgb, params, y, 1, 2)
    t1 = tuned.train(g1, h1)[0]
    _same(t1, plain.train(g1, h1)[0], exact=True)
    nl = int(t1["num_leaves"])
    before = _leaf_sets(tuned, 0, nl)
    default = tuned.launch_shape
    shapes = SHAPES + [default]
    chosen, ms = tuned.time_shapes(shapes, reps=2)
    assert 0 <= chosen < len(shapes)
    assert all(m > 0 for m in ms) and ms[chosen] == min(ms)
    now = tuned.launch_shape
    assert now["partition_ctas"] == shapes[chosen]["partition_ctas"]
    assert now["hist_rows_per_block"] == shapes[chosen]["hist_rows_per_block"]
    # the regrown tree is the last one: its row sets are the partition's
    for ra, rb in zip(before, _leaf_sets(tuned, 0, nl)):
        assert np.array_equal(ra, rb)
    # later trees are those of a learner that was never tuned
    _same(tuned.train(g2, h2)[0], plain.train(g2, h2)[0], exact=True)


def test_launch_shape_errors(lgb):
    X, y = _data(20_000, seed=4)
    params = _params("quantized")
    ds = binned_dataset(lgb, X, y, params)
    learner = lgb.Learner(ds, params)
    before = learner.launch_shape
    for bad in ({"partition_ctas": 0}, {"hist_ctas": 70000}, {"hist_rows_per_block": 16}):
        with pytest.raises(lgb.LightGBMError, match="launch shape"):
            learner.launch_shape = dict(before, **bad)
    assert learner.launch_shape == before
    with pytest.raises(lgb.LightGBMError, match="train first"):
        learner.time_shapes([before])
    persistent = lgb.Learner(ds, dict(params, persistent_grow=True))
    g, h = _grads(lgb, params, y, 1, 5)
    persistent.train(g, h)
    with pytest.raises(lgb.LightGBMError, match="persistent"):
        persistent.time_shapes([before])


@pytest.mark.parametrize("form", ["quantized", "f64"])
def test_wide_scan_grows_the_same_trees(lgb, monkeypatch, form):
    """The register-capped scan (LGBM_B200_SCAN_WIDE, chosen when a step's
    scans span several waves) against the default one, numerical and
    categorical features."""
    X, y = _data(60_000, seed=5)
    rng = np.random.default_rng(6)
    X[:, 18] = rng.integers(0, 12, len(y))
    X[:, 19] = rng.integers(0, 40, len(y))
    y = np.where(np.isin(X[:, 19], [3, 7, 11, 20]), 1.0 - y, y).astype(np.float32)
    params = dict(_params(form), max_cat_to_onehot=4)
    ds = binned_dataset(lgb, X, y, params, categorical=[18, 19])
    monkeypatch.setenv("LGBM_B200_SCAN_WIDE", "0")
    base = lgb.Learner(ds, params)
    monkeypatch.setenv("LGBM_B200_SCAN_WIDE", "1")
    wide = lgb.Learner(ds, params)
    categorical = False
    for it in range(2):
        g, h = _grads(lgb, params, y, 1, 300 + it)
        a = base.train(g, h)[0]
        b = wide.train(g, h)[0]
        _same(a, b, exact=form == "quantized")
        categorical |= bool(np.any(np.asarray(a["decision_type"]) & 1))
    assert categorical  # the categorical scan ran in both variants


@pytest.mark.parametrize("groups", ["2", "3", "4"])
def test_lane_groups_per_tile_grow_the_same_trees(lgb, monkeypatch, groups):
    """The quantized histogram's 32-feature lane groups per feature tile
    (LGBM_B200_HIST_GROUPS; default 1) change the tiling only: 150 features
    in 5 tiles of one group, or 3 / 2 / 2 tiles of several, grow the same
    trees, exactly."""
    X, y = _data(60_000, f=150, seed=4)
    params = _params("quantized")
    ds = binned_dataset(lgb, X, y, params)
    monkeypatch.setenv("LGBM_B200_HIST_GROUPS", "1")
    base = lgb.Learner(ds, params)
    monkeypatch.setenv("LGBM_B200_HIST_GROUPS", groups)
    other = lgb.Learner(ds, params)
    for it in range(2):
        g, h = _grads(lgb, params, y, 1, 200 + it)
        _same(base.train(g, h)[0], other.train(g, h)[0], exact=True)
