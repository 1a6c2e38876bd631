"""Writes the golden fixtures of this directory: small seeded workloads run
through the CPU oracle (the reference's serial learner restated in C++,
pinned by the reference's own known-answer tests).

The fixtures are committed; `tests/test_golden_oracle.py` checks that the
oracle and the host binning still reproduce them and `tests/test_gpu_golden.py`
checks the CUDA path against them. Regenerate with

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "lightgbm-rust_b200"))
sys.path.insert(0, ROOT)

TREE_FIELDS = ("split_feature", "split_feature_inner", "threshold_in_bin", "threshold", "decision_type",
               "left_child", "right_child", "leaf_value", "leaf_count", "internal_value", "internal_count",
               "cat_boundaries", "cat_threshold")
BIN_FIELDS = ("bins", "num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index",
              "upper_bounds", "ub_offsets", "bin_to_cat", "cat_offsets")


def _rows(rng, n, f, nan_frac):
    X = rng.standard_normal((n, f)).astype(np.float32)
    if nan_frac:
        X[rng.random(X.shape) < nan_frac] = np.nan
    return X


def _binary_label(rng, X):
    Z = np.nan_to_num(X)
    z = Z[:, 0] + Z[:, 1] * Z[:, 2] - 0.5 * Z[:, 3] ** 2 + 0.3 * rng.standard_normal(len(X))
    return (rng.random(len(X)) < 1 / (1 + np.exp(-z))).astype(np.float32)


def cases():
    """(name, user params, X, y, X_test, rounds, categorical columns)."""
    out = []
    rng = np.random.default_rng(100)
    X = _rows(rng, 2000, 10, 0.05)
    out.append(("binary_nan", {"objective": "binary", "num_leaves": 15, "min_data_in_leaf": 20},
                X, _binary_label(rng, X), _rows(rng, 300, 10, 0.05), 8, None))
    rng = np.random.default_rng(101)
    X = _rows(rng, 2000, 10, 0.0)
    out.append(("binary_quantized", {"objective": "binary", "num_leaves": 15, "use_quantized_grad": True,
                                     "num_grad_quant_bins": 4, "seed": 7, "num_threads": 4},
                X, _binary_label(rng, X), _rows(rng, 300, 10, 0.0), 5, None))
    rng = np.random.default_rng(102)
    X = _rows(rng, 3000, 8, 0.02)
    X[:, 6] = rng.integers(0, 10, 3000)
    X[:, 7] = rng.integers(0, 6, 3000)
    W = rng.standard_normal((6, 3))
    s = np.nan_to_num(X[:, :6]) @ W + np.eye(3)[X[:, 6].astype(int) % 3]
    Xt = _rows(rng, 400, 8, 0.02)
    Xt[:, 6] = rng.integers(0, 10, 400)
    Xt[:, 7] = rng.integers(0, 6, 400)
    out.append(("multiclass_categorical", {"objective": "multiclass", "num_class": 3, "num_leaves": 15,
                                           "max_cat_to_onehot": 4, "min_data_per_group": 20},
                X, np.argmax(s, axis=1).astype(np.float32), Xt, 3, [6, 7]))
    rng = np.random.default_rng(103)
    X = _rows(rng, 2500, 10, 0.05)
    y = (np.sin(np.nan_to_num(X[:, 0])) + (np.nan_to_num(X[:, 1]) > 0.3) + 0.1 * rng.standard_normal(2500))
    out.append(("l2_bagging", {"objective": "regression", "num_leaves": 31, "learning_rate": 0.05,
                               "bagging_fraction": 0.8, "bagging_freq": 1, "feature_fraction": 0.8,
                               "min_data_in_leaf": 10},
                X, y.astype(np.float32), _rows(rng, 300, 10, 0.05), 5, None))
    return out


def tree_arrays(trees):
    d = {}
    for i, t in enumerate(trees):
        d[f"t{i}_num_leaves"] = np.int32(t["num_leaves"])
        for k in TREE_FIELDS:
            if k in t:
                d[f"t{i}_{k}"] = np.asarray(t[k])
    return d


def main():
    import lgbm_b200 as lgb
    from oracle import oracle as orc

    for name, params, X, y, Xt, rounds, cat in cases():
        ds = lgb.Dataset(X, y, params=params, categorical_feature=cat)
        b = ds.binned()
        p = lgb.resolve_params(params)
        m = orc.train(p, b, y, rounds)
        out = {"params": np.array(json.dumps(params)), "rounds": np.int32(rounds), "X": X, "y": y, "X_test": Xt,
               "categorical": np.asarray(cat if cat else [], np.int32), "num_trees": np.int32(len(m.trees)),
               "pred_raw": m.predict_raw(Xt), "train_scores": m.scores()}
        for k in BIN_FIELDS:
            out["b_" + k] = np.asarray(b[k])
        out.update(tree_arrays(m.trees))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, len(m.trees), "trees")
    # lambdarank gradients and NDCG over uneven query groups
    rng = np.random.default_rng(104)
    group = rng.integers(1, 40, 60)
    n = int(group.sum())
    label = rng.integers(0, 5, n).astype(np.float32)
    score = rng.standard_normal(n)
    p = lgb.resolve_params({"objective": "lambdarank"})
    g, h = orc.gradients(p, label, score, group)
    ks = np.array([1, 3, 5, 10], np.int32)
    np.savez_compressed(os.path.join(HERE, "lambdarank.npz"), group=group.astype(np.int32), label=label, score=score,
                        grad=g, hess=h, ks=ks, ndcg=orc.ndcg(label, score, group, ks))
    print("lambdarank", n, "rows")


if __name__ == "__main__":
    main()
