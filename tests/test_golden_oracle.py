"""The committed golden fixtures (tests/golden, written by make_golden.py
from the CPU oracle) are reproduced by the host binning and by the oracle:
a change to either that alters a fixture fails here, on the CPU."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["binary_nan", "binary_quantized", "multiclass_categorical", "l2_bagging"]
BIN_FIELDS = ("bins", "num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index",
              "upper_bounds", "ub_offsets", "bin_to_cat", "cat_offsets")
TREE_FIELDS = ("split_feature", "split_feature_inner", "threshold_in_bin", "threshold", "decision_type",
               "left_child", "right_child", "leaf_value", "leaf_count", "internal_value", "internal_count",
               "cat_boundaries", "cat_threshold")


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=a.dtype.kind == "f")


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def golden_binned(d):
    b = {k: d["b_" + k] for k in BIN_FIELDS}
    b["num_data"] = int(d["b_bins"].shape[0])
    b["num_features"] = int(d["b_bins"].shape[1])
    return b


def case_inputs(d):
    params = json.loads(str(d["params"]))
    cat = [int(c) for c in d["categorical"]] or None
    return params, cat


@pytest.mark.parametrize("name", CASES)
def test_host_binning_reproduces_golden(lgb, name):
    d = load(name)
    params, cat = case_inputs(d)
    b = lgb.Dataset(d["X"], d["y"], params=params, categorical_feature=cat).binned()
    for k in BIN_FIELDS:
        assert same(b[k], d["b_" + k]), k


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(lgb, orc, name):
    d = load(name)
    params, _ = case_inputs(d)
    m = orc.train(lgb.resolve_params(params), golden_binned(d), d["y"], int(d["rounds"]))
    assert len(m.trees) == int(d["num_trees"])
    for i, t in enumerate(m.trees):
        assert t["num_leaves"] == int(d[f"t{i}_num_leaves"])
        for k in TREE_FIELDS:
            assert same(t[k], d[f"t{i}_{k}"]), (i, k)
    assert same(m.predict_raw(d["X_test"]), d["pred_raw"])
    assert same(m.scores(), d["train_scores"])


def test_oracle_lambdarank_golden(lgb, orc):
    d = load("lambdarank")
    p = lgb.resolve_params({"objective": "lambdarank"})
    g, h = orc.gradients(p, d["label"], d["score"], d["group"])
    assert np.array_equal(g, d["grad"]) and np.array_equal(h, d["hess"])
    assert np.array_equal(orc.ndcg(d["label"], d["score"], d["group"], d["ks"]), d["ndcg"])
