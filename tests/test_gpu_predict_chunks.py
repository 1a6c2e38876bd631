"""Batched prediction from host rows (lgbm_b200_predict, predict.rs:231):
the rows stream through the device in chunks over two pinned buffers. The
same forest predicts bit for bit the same with one chunk and with several,
a partial last chunk included, and equals the oracle's prediction."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(n, f=12, seed=0, classes=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    z = np.nan_to_num(X[:, 0] + X[:, 1] * X[:, 2]) + 0.3 * rng.standard_normal(n)
    if classes:
        return X, np.digitize(z, np.quantile(z, np.linspace(0, 1, classes + 1)[1:-1])).astype(np.float32)
    return X, (rng.random(n) < 1 / (1 + np.exp(-z))).astype(np.float32)


@pytest.mark.parametrize("classes", [0, 3])
def test_predict_chunks_match_one_chunk_and_oracle(lgb, orc, monkeypatch, classes):
    X, y = _data(20_000, seed=31, classes=classes)
    params = {"objective": "multiclass", "num_class": classes} if classes else {"objective": "binary"}
    params.update(num_leaves=15, min_data_in_leaf=20)
    ds = lgb.Dataset(X, y, params=params)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, 8)
    bst = lgb.Booster(params)
    bst.trees = [dict(t, leaf_parent=np.zeros(t["num_leaves"], np.int32),
                      cat_boundaries_inner=np.zeros(1, np.int32), cat_threshold_inner=np.zeros(0, np.uint32))
                 for t in om.trees]
    Xt, _ = _data(5_500, seed=32, classes=classes)
    whole = bst.predict(Xt, raw_score=True)
    monkeypatch.setenv("LGBM_B200_PREDICT_CHUNK_ROWS", "1000")  # 6 chunks, the last of 500 rows
    bst._forest = None
    chunked = bst.predict(Xt, raw_score=True)
    assert np.array_equal(whole, chunked)
    want = om.predict_raw(Xt)
    assert np.array_equal(np.asarray(chunked).reshape(want.shape), want)


def test_predict_more_than_64_classes_matches_oracle(lgb, orc):
    """num_tree_per_iteration above 64: every class sums its own trees in
    model order (no fixed-size per-class array), bit-exact with the oracle."""
    k = 70
    rng = np.random.default_rng(33)
    n = 7_000
    X = rng.standard_normal((n, 6)).astype(np.float32)
    y = rng.integers(0, k, n).astype(np.float32)
    params = {"objective": "multiclass", "num_class": k, "num_leaves": 4, "min_data_in_leaf": 5}
    ds = lgb.Dataset(X, y, params=params)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, 2)
    assert len(om.trees) == 2 * k
    bst = lgb.Booster(params)
    bst.trees = [dict(t, leaf_parent=np.zeros(t["num_leaves"], np.int32),
                      cat_boundaries_inner=np.zeros(1, np.int32), cat_threshold_inner=np.zeros(0, np.uint32))
                 for t in om.trees]
    Xt = rng.standard_normal((3_000, 6)).astype(np.float32)
    got = bst.predict(Xt, raw_score=True)
    want = om.predict_raw(Xt)
    assert got.shape == want.shape == (3_000, k)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("ncol", [3, 136, 300])
def test_predict_row_staging_widths(lgb, orc, ncol):
    """Rows staged in shared memory (up to 223 features, vector loads when
    the row width is a multiple of 4) and read in place above that: all
    bit-exact with the oracle."""
    rng = np.random.default_rng(34 + ncol)
    n = 4_000
    X = rng.standard_normal((n, ncol)).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    X[rng.random(X.shape) < 0.05] = 0.0
    X[rng.random(X.shape) < 0.01] = 1e-38  # below the zero threshold: read as 0
    z = np.nan_to_num(X[:, 0]) + np.nan_to_num(X[:, ncol - 1]) * np.nan_to_num(X[:, ncol // 2])
    y = (z + 0.3 * rng.standard_normal(n) > 0).astype(np.float32)
    params = {"objective": "binary", "num_leaves": 15, "min_data_in_leaf": 10}
    ds = lgb.Dataset(X, y, params=params)
    om = orc.train(lgb.resolve_params(params), ds.binned(), y, 6)
    bst = lgb.Booster(params)
    bst.trees = [dict(t, leaf_parent=np.zeros(t["num_leaves"], np.int32),
                      cat_boundaries_inner=np.zeros(1, np.int32), cat_threshold_inner=np.zeros(0, np.uint32))
                 for t in om.trees]
    Xt = X[:1_537]  # a partial last CTA of rows
    assert np.array_equal(bst.predict(Xt, raw_score=True), om.predict_raw(Xt)[:, 0])
