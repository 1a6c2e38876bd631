"""The host-side binning (the Rust host's Dataset stand-in) against the
reference's binning known answers (crates/lgbm-core/src/binning.rs:704-779),
and the stored group values of a dense single-feature group
(feature_group.rs:144-154). No GPU needed."""
import numpy as np
import pytest

from conftest import binned_dataset

KZ = float(np.float32(1e-35))


def _one_column(lgb, vals, n_zero=0, max_bin=255, categorical=False):
    x = np.concatenate([np.asarray(vals, np.float64), np.zeros(n_zero)]).astype(np.float32).reshape(-1, 1)
    params = {"max_bin": max_bin, "min_data_in_bin": 3, "feature_pre_filter": False, "min_data_in_leaf": 1}
    ds = binned_dataset(lgb, x, np.zeros(len(x), np.float32), params, categorical=[0] if categorical else None)
    return ds.binned(), x


def test_small_distinct_values_get_midpoint_bounds(lgb):  # binning.rs:704-716
    vals = np.repeat(np.arange(1, 11, dtype=np.float64), 5)
    b, _ = _one_column(lgb, vals)
    assert b["missing_type"][0] == 0
    ub = b["upper_bounds"]
    assert ub[0] == KZ
    assert ub[1] == np.nextafter(1.5, np.inf)
    assert ub[-1] == np.inf


def test_nan_gets_last_bin(lgb):  # binning.rs:718-727
    vals = np.concatenate([np.arange(1, 51, dtype=np.float64), [np.nan, np.nan]])
    b, x = _one_column(lgb, vals)
    assert b["missing_type"][0] == 2
    assert np.isnan(b["upper_bounds"][-1])
    nb = int(b["num_bin"][0])
    mfb = int(b["most_freq_bin"][0])
    raw = b["bins"][-1, 0]  # a NaN row: bin num_bin - 1
    bin_ = mfb if raw == 0 else raw - 1 + (mfb == 0)
    assert bin_ == nb - 1


def test_greedy_respects_max_bin(lgb):  # binning.rs:729-737
    vals = np.sin(np.arange(10000) * 0.37) + 2.0
    b, _ = _one_column(lgb, vals, max_bin=16)
    assert b["num_bin"][0] <= 16
    assert np.all(np.diff(b["upper_bounds"]) > 0)


def test_categorical_bins_by_count(lgb):  # binning.rs:739-761
    vals = np.concatenate([np.full(30, 3.0), np.full(20, 1.0), np.full(10, 2.7), np.full(5, -1.0)])
    b, x = _one_column(lgb, vals, n_zero=15, categorical=True)
    assert list(b["bin_to_cat"]) == [-1, 3, 1, 0, 2]
    assert b["missing_type"][0] == 2
    assert b["default_bin"][0] == 3


def test_constant_feature_is_trivial(lgb):  # binning.rs:775-779
    x = np.zeros((100, 2), np.float32)
    x[:, 1] = np.arange(100)
    ds = binned_dataset(lgb, x, np.zeros(100, np.float32), {"min_data_in_leaf": 1})
    b = ds.binned()
    assert b["num_features"] == 1
    assert list(b["real_index"]) == [1]


def test_group_values_match_value_to_bin(lgb):
    """Stored value = 0 for the most frequent bin, else bin - (mfb == 0) + 1."""
    rng = np.random.default_rng(0)
    X = rng.standard_normal((5000, 4)).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    X[:, 3] = rng.integers(0, 5, 5000)
    ds = binned_dataset(lgb, X, np.zeros(5000, np.float32), {})
    b = ds.binned()
    for f in range(b["num_features"]):
        ub = b["upper_bounds"][b["ub_offsets"][f]: b["ub_offsets"][f + 1]]
        nb, mfb, mt = int(b["num_bin"][f]), int(b["most_freq_bin"][f]), int(b["missing_type"][f])
        col = X[:, b["real_index"][f]].astype(np.float64)
        want = np.empty(len(col), np.int64)
        for i, v in enumerate(col):
            if np.isnan(v) and mt == 2:
                want[i] = nb - 1
                continue
            v = 0.0 if np.isnan(v) else v
            hi = nb - 1 - (1 if mt == 2 else 0)
            want[i] = min(int(np.searchsorted(ub[:hi], v, side="left")), hi)
        stored = np.where(want == mfb, 0, want - (1 if mfb == 0 else 0) + 1)
        assert np.array_equal(b["bins"][:, f], stored), f


def test_bundleable_features_rejected(lgb):
    """Sparse features that exclusive feature bundling could merge are out of scope."""
    X = np.zeros((2000, 2), np.float32)
    X[:100, 0] = 1.0
    X[100:200, 1] = 2.0
    with pytest.raises(lgb.LightGBMError):
        binned_dataset(lgb, X, np.zeros(2000, np.float32), {"min_data_in_leaf": 1})


@pytest.mark.parametrize("cfg,scale", [("config0", 1.0), ("config1", 0.02), ("config2", 0.003), ("config3", 0.005),
                                       ("config4", 0.003)])
def test_product_binning_equals_the_oracle_restatement(lgb, orc, cfg, scale):
    """The product's host binning (host_dataset.cpp) and the oracle's own
    restatement of binning.rs / dataset.rs (oracle/binning.cpp) give the same
    bin matrix, bin mappers and thresholds on each workload's generator, and
    the same for the held-out rows binned with the training mappers."""
    from lgbm_b200 import synthetic as syn

    d = getattr(syn, cfg)(scale=scale)
    params = d["params"]
    cats = d.get("categorical")
    p = lgb.resolve_params(params)
    ds = lgb.Dataset(d["X"], d["y"], params=params, categorical_feature=cats)
    od = orc.Dataset(d["X"], p, categorical=cats)
    b, ob = ds.binned(), od.binned()
    assert set(b) == set(ob)
    for k in b:
        assert np.array_equal(np.asarray(b[k]), np.asarray(ob[k]), equal_nan=True), k
    if "X_valid" in d:
        dv = lgb.Dataset(d["X_valid"], d["y_valid"], params=params, reference=ds)
        odv = orc.Dataset(d["X_valid"], p, reference=od)
        assert np.array_equal(dv.binned()["bins"], odv.binned()["bins"])


def test_oracle_feature_infos_format(orc, lgb):
    """Dataset::feature_infos (dataset.rs:770): [min:max] with %.17g for a
    numerical feature, the categories of each bin joined by ':' for a
    categorical one, none for a feature left out as trivial."""
    rng = np.random.default_rng(5)
    n = 5000
    X = np.stack([rng.standard_normal(n), np.full(n, 3.0), rng.integers(0, 4, n)], axis=1).astype(np.float32)
    p = lgb.resolve_params({})
    od = orc.Dataset(X, p, categorical=[2])
    info = od.feature_infos
    assert info[0] == "[%.17g:%.17g]" % (float(X[:, 0].min()), float(X[:, 0].max()))
    assert info[1] == "none"
    cats = info[2].split(":")
    assert cats[0] == "-1" and sorted(cats[1:]) == ["0", "1", "2", "3"]
