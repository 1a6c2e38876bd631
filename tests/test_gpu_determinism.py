"""Run-to-run determinism and the partition contract, through the C ABI.

- The quantized form with FP64 leaf renewal (quant_train_renew_leaf) grows
  bit-identical trees and scores when the same model is trained twice: its
  histograms are integer sums, and the renewal's FP64 sums are reduced in a
  fixed order (per-warp segment sums added in warp order), not by atomics.
- partition() returns each leaf's rows in ascending order, the reference's
  partition_is_stable known-answer test (learner/tests.rs:45-63), and the
  leaf row lists equal the oracle's element for element.
"""
import numpy as np
import pytest

from conftest import binned_dataset

pytestmark = pytest.mark.gpu


def _binary_10m_form(n, seed):
    """The 10M-row binary workload's generator at n rows: 21 N(0,1)
    features and 7 heavy-tailed products / ratios of them."""
    import lgbm_b200.synthetic as syn

    d = syn.config2(scale=n / 10_000_000, seed=seed)
    return d["X"], d["y"]


def _train_twice(lgb, X, y, params, rounds):
    out = []
    for _ in range(2):
        ds = lgb.Dataset(X, y, params=params)
        bst = lgb.train(params, ds, rounds)
        out.append(bst)
    return out


def test_quantized_renewal_is_bit_reproducible(lgb):
    X, y = _binary_10m_form(200_000, seed=41)
    params = {"objective": "binary", "num_leaves": 255, "learning_rate": 0.1, "use_quantized_grad": True,
              "num_grad_quant_bins": 4, "quant_train_renew_leaf": True, "num_threads": 16, "seed": 3}
    a, b = _train_twice(lgb, X, y, params, 12)
    assert a.num_trees() == b.num_trees() == 12
    for ta, tb in zip(a.trees, b.trees):
        for k in ("split_feature", "threshold_in_bin", "left_child", "right_child", "leaf_count"):
            assert np.array_equal(ta[k], tb[k]), k
        # bit-identical FP64 leaf values (renewed from FP64 gradient sums)
        assert np.array_equal(ta["leaf_value"].view(np.int64), tb["leaf_value"].view(np.int64))
    assert np.array_equal(a.scores().view(np.int64), b.scores().view(np.int64))


def test_partition_is_stable_through_the_c_abi(lgb):
    """learner/tests.rs:45-63: x0 = i / n decides the label, x1 = (37 i) mod 11
    is noise; 4 leaves, min_data_in_leaf 3, gradients ((7919 i) mod 13) - 6."""
    n = 100
    i = np.arange(n)
    X = np.stack([i / n, (i * 37) % 11], axis=1).astype(np.float32)
    y = np.where(i / n < 0.5, -1.0, 1.0).astype(np.float32)
    params = {"objective": "regression", "num_leaves": 4, "min_data_in_leaf": 3}
    ds = binned_dataset(lgb, X, y, params)
    learner = lgb.Learner(ds, params)
    g = (((i * 7919) % 13) - 6).astype(np.float32)
    h = np.ones(n, np.float32)
    tree = learner.train(g, h)[0]
    beg, cnt, idx = learner.partition(0, tree["num_leaves"])
    seen = 0
    for leaf in range(tree["num_leaves"]):
        rows = idx[beg[leaf]: beg[leaf] + cnt[leaf]]
        assert np.all(np.diff(rows.astype(np.int64)) > 0), f"leaf {leaf} indices not increasing"
        seen += len(rows)
    assert seen == n


@pytest.mark.parametrize("form", ["f64", "quantized"])
def test_partition_lists_equal_the_oracle(lgb, orc, form):
    """Every leaf's row list, in order, equals the oracle's (the reference's
    stable partition) after a 255-leaf tree on 50k rows."""
    X, y = _binary_10m_form(50_000, seed=42)
    params = {"objective": "binary", "num_leaves": 255, "min_data_in_leaf": 20, "hist_precision": form,
              "num_threads": 16}
    ds = binned_dataset(lgb, X, y, params)
    b = ds.binned()
    p = lgb.resolve_params(params)
    g, h = orc.gradients(p, y, np.zeros(len(y)))
    learner = lgb.Learner(ds, params)
    gt = learner.train(g, h)[0]
    om = orc.train_trees(p, b, g, h)
    ot = om.trees[0]
    assert np.array_equal(gt["split_feature"], ot["split_feature"])
    beg, cnt, idx = learner.partition(0, gt["num_leaves"])
    obeg, ocnt, oidx = orc.partition(om, ot["num_leaves"], len(y))
    for leaf in range(gt["num_leaves"]):
        assert np.array_equal(idx[beg[leaf]: beg[leaf] + cnt[leaf]], oidx[obeg[leaf]: obeg[leaf] + ocnt[leaf]]), leaf
