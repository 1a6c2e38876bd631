"""The booster's captured iteration (gradients, quantization, the tree and
the score updates replayed as one CUDA graph from the second iteration on)
against the same boosting run launch by launch (LGBM_B200_ITER_GRAPH=0).

Quantized runs match exactly (integer histograms, the same quantization
offsets drawn in the same order); FP64 runs match within the FP64 bars
(histogram atomics add in another order). A launch-shape change mid-run
makes the booster capture its iteration again."""
import numpy as np
import pytest

from conftest import binned_dataset

pytestmark = pytest.mark.gpu


def _data(n, f=16, seed=0, classes=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    X[rng.random(X.shape) < 0.03] = np.nan
    z = np.nan_to_num(X[:, 0] + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2) + 0.3 * rng.standard_normal(n)
    if classes:
        y = np.digitize(z, np.quantile(z, np.linspace(0, 1, classes + 1)[1:-1])).astype(np.float32)
    else:
        y = (rng.random(n) < 1 / (1 + np.exp(-z))).astype(np.float32)
    return X, y


def _ranking(nq, f=12, seed=0):
    rng = np.random.default_rng(seed)
    group = np.clip(rng.geometric(1 / 20, nq), 1, 200).astype(np.int32)
    n = int(group.sum())
    X = rng.standard_normal((n, f)).astype(np.float32)
    s = X[:, 0] + 0.5 * X[:, 1] + 0.5 * rng.standard_normal(n)
    y = np.digitize(s, np.quantile(s, [0.5, 0.75, 0.9, 0.97])).astype(np.float32)
    return X, y, group


CASES = {
    "binary_quantized_valid": dict(params={"objective": "binary", "num_leaves": 31, "use_quantized_grad": True,
                                           "num_grad_quant_bins": 4, "quant_train_renew_leaf": True,
                                           "num_threads": 8, "seed": 3}, exact=True, valid=True),
    "l2_f64_feature_fraction": dict(params={"objective": "regression", "num_leaves": 31, "feature_fraction": 0.7,
                                            "feature_fraction_seed": 5}, exact=False, valid=False),
    "multiclass_quantized": dict(params={"objective": "multiclass", "num_class": 3, "num_leaves": 15,
                                         "use_quantized_grad": True, "num_threads": 8, "seed": 4},
                                 exact=True, valid=False),
    "lambdarank_quantized": dict(params={"objective": "lambdarank", "num_leaves": 15, "use_quantized_grad": True,
                                         "num_threads": 8, "seed": 5}, exact=True, valid=False),
}


def _build(lgb, case, monkeypatch, graph):
    c = CASES[case]
    params = dict(c["params"])
    monkeypatch.setenv("LGBM_B200_ITER_GRAPH", "1" if graph else "0")
    if case.startswith("lambdarank"):
        X, y, group = _ranking(300, seed=7)
        ds = lgb.Dataset(X, y, group=group, params=params)
        ds.construct(params)
        return lgb.Booster(params, ds)
    X, y = _data(40_000, seed=1, classes=int(params.get("num_class", 0)))
    if params["objective"] == "regression":
        y = (np.nan_to_num(X[:, 0]) + 0.1 * np.nan_to_num(X[:, 5])).astype(np.float32)
    ds = binned_dataset(lgb, X, y, params)
    dv = None
    if c["valid"]:
        Xv, yv = _data(8_000, seed=2)
        dv = binned_dataset(lgb, Xv, yv, params, reference=ds)
    return lgb.Booster(params, ds, dv)


def _same_tree(a, b, exact):
    assert a["num_leaves"] == b["num_leaves"]
    for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child", "leaf_count"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    for k in ("leaf_value", "internal_value"):
        if exact:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
        else:
            np.testing.assert_allclose(a[k], b[k], rtol=1e-9, atol=1e-12, err_msg=k)


@pytest.mark.parametrize("case", sorted(CASES))
def test_iteration_graph_matches_launch_by_launch(lgb, monkeypatch, case):
    exact = CASES[case]["exact"]
    plain = _build(lgb, case, monkeypatch, graph=False)
    graphed = _build(lgb, case, monkeypatch, graph=True)
    for it in range(7):
        if it == 4 and exact:  # the captured iteration is captured again with the new grids
            graphed.learner.launch_shape = {"partition_ctas": 20, "hist_ctas": 16, "hist_rows_per_block": 256}
        assert plain.update() == graphed.update()
    assert plain.num_trees() == graphed.num_trees() > 0
    for a, b in zip(plain.trees, graphed.trees):
        _same_tree(a, b, exact)
    for valid in ([False, True] if CASES[case]["valid"] else [False]):
        sa, sb = plain.scores(valid), graphed.scores(valid)
        if exact:
            assert np.array_equal(sa, sb)
        else:
            np.testing.assert_allclose(sa, sb, rtol=1e-9, atol=1e-12)
