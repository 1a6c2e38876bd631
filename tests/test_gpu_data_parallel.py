"""The data-parallel learner (lgbm_b200_learner_set_data_parallel) against one
learner on all rows, through the C ABI. Two ranks run as two processes on one
GPU; their reductions go through host memory over gloo, so no kernel of one
rank ever waits on the other's. The rows are sharded unevenly.

- quantized histograms: integer sums are order-free, so every tree equals
  the single learner's bit for bit (structure, gains, leaf values);
- quantized with FP64 leaf renewal, and FP64 histograms: structure exact,
  gains and leaf values within tests/tolerances.toml (FP64 sums are added in
  another order).
"""
import json
import os
import pickle
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import TOL, binned_dataset, within

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 12)).astype(np.float32)
    X[rng.random(X.shape) < 0.03] = np.nan
    z = np.nan_to_num(X[:, 0] + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2) + 0.3 * rng.standard_normal(n)
    y = (rng.random(n) < 1 / (1 + np.exp(-z))).astype(np.float32)
    return X, y


@pytest.mark.parametrize("form,renew", [("quantized", False), ("quantized", True), ("f64", False)])
def test_two_ranks_grow_the_single_learners_trees(lgb, orc, tmp_path, form, renew):
    n = 30_000
    X, y = _data(n, seed=51)
    params = {"objective": "binary", "num_leaves": 63, "min_data_in_leaf": 20, "hist_precision": form,
              "num_threads": 8, "seed": 9, "quant_train_renew_leaf": renew}
    p = lgb.resolve_params(params)
    rng = np.random.default_rng(52)
    grads = [orc.gradients(p, y, rng.standard_normal(n) * s) for s in (0.0, 0.5, 1.5)]
    ds = binned_dataset(lgb, X, y, params)
    single = lgb.Learner(ds, params)
    want = [single.train(g, h)[0] for g, h in grads]
    bounds = np.array([0, 13_001, n])  # uneven shards
    np.savez(tmp_path / "case.npz", X=X, y=y, g=np.stack([g for g, _ in grads]),
             h=np.stack([h for _, h in grads]), bounds=bounds)
    (tmp_path / "params.json").write_text(json.dumps(params))
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "dp_rank.py"), str(r), "2", str(port),
                               str(tmp_path)]) for r in range(2)]
    try:
        rcs = [pr.wait(timeout=300) for pr in procs]
    finally:
        for pr in procs:
            if pr.poll() is None:
                pr.kill()
    assert rcs == [0, 0]
    ranks = [pickle.load(open(tmp_path / f"rank{r}.pkl", "rb")) for r in range(2)]
    for got in ranks:
        assert len(got) == len(want)
        for a, b in zip(got, want):
            assert a["num_leaves"] == b["num_leaves"]
            for k in ("split_feature", "threshold_in_bin", "decision_type", "left_child", "right_child",
                      "leaf_count", "internal_count", "leaf_depth"):
                assert np.array_equal(a[k], b[k]), k
            if form == "quantized" and not renew:
                assert np.array_equal(a["leaf_value"], b["leaf_value"])
                assert np.array_equal(a["split_gain_f64"], b["split_gain_f64"])
            else:
                assert within(a["leaf_value"], b["leaf_value"], "leaf_value")
                g = TOL["split_gain"]
                np.testing.assert_allclose(a["split_gain_f64"], b["split_gain_f64"], rtol=g["rtol"], atol=0)
    # both ranks grew the same trees
    for a, b in zip(ranks[0], ranks[1]):
        assert np.array_equal(a["leaf_value"], b["leaf_value"])
