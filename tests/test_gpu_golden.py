"""The CUDA path against the committed golden fixtures (tests/golden): the
same workloads boosted on the device through the public API give the
fixtures' trees and raw predictions."""
import json
import os

import numpy as np
import pytest

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

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["binary_nan", "binary_quantized", "multiclass_categorical", "l2_bagging"]
EXACT = ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child", "leaf_count",
         "cat_boundaries", "cat_threshold")


@pytest.mark.parametrize("name", CASES)
def test_device_boosting_matches_golden(lgb, name):
    d = np.load(os.path.join(GOLD, name + ".npz"))
    params = json.loads(str(d["params"]))
    cat = [int(c) for c in d["categorical"]] or None
    bst = lgb.train(params, lgb.Dataset(d["X"], d["y"], params=params, categorical_feature=cat), int(d["rounds"]))
    assert bst.num_trees() == int(d["num_trees"])
    for i, t in enumerate(bst.trees):
        assert t["num_leaves"] == int(d[f"t{i}_num_leaves"]), i
        for k in EXACT:
            assert np.array_equal(np.asarray(t[k]), d[f"t{i}_{k}"]), (i, k)
        # device gradients are within 1 ulp of the oracle's, so FP64 sums agree to ~1e-7 relative
        np.testing.assert_allclose(t["leaf_value"], d[f"t{i}_leaf_value"], rtol=1e-7, atol=1e-12,
                                   err_msg=f"tree {i}")
    raw = bst.predict(d["X_test"], raw_score=True).reshape(d["pred_raw"].shape)
    np.testing.assert_allclose(raw, d["pred_raw"], rtol=1e-6, atol=1e-9)


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_device_lambdarank_gradients_match_golden(lgb):
    d = np.load(os.path.join(GOLD, "lambdarank.npz"))
    g, h = lgb.gradients({"objective": "lambdarank"}, d["label"], d["score"], group=d["group"])
    # the pair loop runs in the reference's order, so sums are exact; the
    # final normalisation's log2 is CUDA's (within 1 ulp of the host's)
    assert _ulps(g, d["grad"]).max() <= 1 and _ulps(h, d["hess"]).max() <= 1
    assert np.mean(_ulps(g, d["grad"]) == 0) > 0.9
