"""Test configuration: paths, the `gpu` marker, shared fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's known
answers, the host-side code and the C ABI's exports; GPU tests (-m gpu)
compare the CUDA path with the oracle through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "lightgbm-rust_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """liblgbm_b200.so and the oracle, built in-tree (cached by mtime)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("lgbm_b200_build", os.path.join(ROOT, "lightgbm-rust_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)

    if not os.environ.get("LGBM_B200_SKIP_BUILD"):
        b.build()
    from oracle import oracle

    oracle.build()
    return True


@pytest.fixture(scope="session")
def lgb(built):
    import lgbm_b200

    return lgbm_b200


@pytest.fixture(scope="session")
def orc(built):
    from oracle import oracle

    return oracle


def binned_dataset(lgb, X, y=None, params=None, reference=None, categorical=None):
    ds = lgb.Dataset(X, label=y, params=params, reference=reference, categorical_feature=categorical)
    ds.construct(params)
    return ds


def tolerances():
    """The parity bars of tests/tolerances.toml."""
    import tomllib

    with open(os.path.join(ROOT, "tests", "tolerances.toml"), "rb") as f:
        return tomllib.load(f)


TOL = tolerances()


def within(got, want, section):
    """|got - want| <= atol + rtol * |want| under TOL[section] (NaN == NaN)."""
    t = TOL[section]
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    ok = np.abs(got - want) <= t.get("atol", 0.0) + t["rtol"] * np.abs(want)
    return bool(np.all(ok | (np.isnan(got) & np.isnan(want))))


def compare_boosted_trees(gpu_trees, oracle_model, leaf_section="leaf_value"):
    """Walk two boosting runs tree by tree: the structure must be exact, the
    FP64 split gains within TOL["split_gain"] of the oracle's trace and the
    leaf values within TOL[leaf_section]. At the first split where the two
    pick different candidates, the pick must be a gain tie (the two gains
    within TOL["split_gain"]["tie_rtol"]); later trees legitimately differ
    and are not compared. Returns (identical trees, tie or None) where tie =
    (tree, node, gpu gain, oracle gain)."""
    g = TOL["split_gain"]
    for i, (a, o) in enumerate(zip(gpu_trees, oracle_model.trees)):
        _, feat, thr, gains = oracle_model.trace(i)
        nn = min(a["num_leaves"], o["num_leaves"]) - 1
        for j in range(nn):
            ga = float(a["split_gain_f64"][j])
            same = a["split_feature"][j] == o["split_feature"][j] and a["threshold_in_bin"][j] == o["threshold_in_bin"][j]
            if not same:
                assert abs(ga - gains[j]) <= g["tie_rtol"] * abs(gains[j]), (
                    f"tree {i} node {j}: different split without a gain tie", ga, gains[j])
                return i, (i, j, ga, float(gains[j]))
            assert abs(ga - gains[j]) <= g["atol"] + g["rtol"] * abs(gains[j]), (i, j, ga, gains[j])
        assert a["num_leaves"] == o["num_leaves"], (i, a["num_leaves"], o["num_leaves"])
        for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child", "leaf_count",
                  "internal_count", "leaf_depth"):
            assert np.array_equal(np.asarray(a[k]), np.asarray(o[k])), (i, k)
        for k in ("leaf_value", "leaf_weight", "internal_value", "internal_weight"):
            assert within(a[k], o[k], leaf_section), (i, k, np.max(np.abs(a[k] - o[k])))
    return len(gpu_trees), None
