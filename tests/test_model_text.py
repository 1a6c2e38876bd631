"""The model text writer of the host side (lgbm_b200/model_text.py) against
the oracle's restatement of io.rs:13-85, tree.rs:718-773 and fmt.rs, on the
oracle's own models: the same trees give the same bytes. No GPU needed; the
GPU model's text is compared with the oracle's in test_gpu_config0.py."""
import numpy as np
import pytest

from lgbm_b200 import model_text


def _oracle_model(lgb, orc, params, X, y, rounds, categorical=None, group=None):
    p = lgb.resolve_params(params)
    od = orc.Dataset(X, p, categorical=categorical)
    om = orc.train(p, od.binned(), y, rounds, group=group)
    return p, od, om


@pytest.mark.parametrize("case", ["binary", "multiclass_categorical", "regression_nan", "lambdarank"])
def test_writer_matches_the_oracle_text(lgb, orc, case):
    rng = np.random.default_rng(7)
    n = 3000
    X = rng.standard_normal((n, 6)).astype(np.float32)
    group = None
    cats = None
    if case == "binary":
        params = {"objective": "binary", "num_leaves": 15}
        y = (X[:, 0] + X[:, 1] * X[:, 2] > 0).astype(np.float32)
    elif case == "multiclass_categorical":
        X[:, 5] = rng.integers(0, 8, n)
        cats = [5]
        params = {"objective": "multiclass", "num_class": 3, "num_leaves": 7, "max_cat_to_onehot": 4}
        y = ((X[:, 0] > 0).astype(int) + (X[:, 5] > 4)).astype(np.float32)
    elif case == "regression_nan":
        X[rng.random(X.shape) < 0.1] = np.nan
        params = {"objective": "regression", "num_leaves": 31, "learning_rate": 0.05}
        y = np.nan_to_num(X[:, 0]).astype(np.float32) + 0.1 * rng.standard_normal(n).astype(np.float32)
    else:
        group = np.full(n // 30, 30, np.int32)
        params = {"objective": "lambdarank", "num_leaves": 7}
        y = np.clip(np.round(X[:, 0] + 1.5), 0, 4).astype(np.float32)
    p, od, om = _oracle_model(lgb, orc, params, X, y, 5, categorical=cats, group=group)
    want = om.model_to_string(X.shape[1], od.feature_infos)
    ntpi = int(p["num_class"]) if p["objective"] == "multiclass" else 1
    got = model_text.model_to_string(p, om.trees, [t["shrinkage"] for t in om.trees], ntpi, X.shape[1],
                                     od.feature_infos)
    assert got == want
    assert want.startswith("tree\nversion=v4\n")
    assert "\nend of trees\n" in want and "\nfeature_importances:\n" in want


def test_number_formatting_is_c_printf():
    """fmt.rs fmt_g: %g with 6 and 17 significant digits, C's exponent form."""
    assert model_text.fmt_g(0.1, 17) == "0.10000000000000001"
    assert model_text.fmt_g(1e-5, 6) == "1e-05"
    assert model_text.fmt_g(123456789.0, 6) == "1.23457e+08"
    assert model_text.fmt_g(-0.0, 6) == "-0"
    assert model_text.fmt_g(float("inf"), 17) == "inf"
    assert model_text.fmt_g(-1e308 * 10, 6) == "-inf"
    assert model_text.fmt_g(2.5, 6) == "2.5"
