"""Rows binned on the device (lgbm_b200_dataset_create_device and
..._create_valid_device) against the host build: the same dataset, byte for
byte, over numerical columns with NaN, zeros, heavy tails and infinities,
categorical columns with unseen, negative and NaN values, both missing-value
settings, and a matrix wide enough to stream through several chunks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrix(n, seed, wide=False):
    rng = np.random.default_rng(seed)
    cols = [
        rng.standard_normal(n),
        rng.lognormal(0.0, 1.0, n),
        rng.integers(0, 16, n).astype(np.float64),
        rng.standard_cauchy(n),
        np.where(rng.random(n) < 0.3, 0.0, rng.standard_normal(n)),  # exact zeros
        rng.choice(50, n, p=(1.0 / np.arange(1, 51) ** 1.2) / np.sum(1.0 / np.arange(1, 51) ** 1.2)).astype(
            np.float64),  # categorical, Zipf
    ]
    if wide:
        cols += [rng.standard_normal(n) * (k + 1) for k in range(40)]
    X = np.stack(cols, axis=1).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    X[rng.random(n) < 0.001, 3] = np.inf
    X[rng.random(n) < 0.001, 3] = -np.inf
    return X


def _same(a, b):
    for k in ("bins", "num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index",
              "upper_bounds", "bin_to_cat", "ub_offsets", "cat_offsets"):
        assert np.array_equal(a[k], b[k], equal_nan=True) if a[k].dtype.kind == "f" else np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("flags", [{}, {"zero_as_missing": True}, {"use_missing": False}])
def test_device_binning_matches_host(lgb, flags):
    X = _matrix(60000, 1)
    params = dict({"max_bin": 255, "categorical_feature": [5]}, **flags)
    host = lgb.Dataset(X, params=params).construct()
    dev = lgb.Dataset(X, params=dict(params, device_binning=True)).construct()
    _same(host.binned(), dev.binned())
    # held-out rows with categories never seen, negative and NaN ones
    Xv = _matrix(20000, 2)
    Xv[:500, 5] = 77.0
    Xv[500:1000, 5] = -3.0
    hv = lgb.Dataset(Xv, reference=host).construct()
    dv = lgb.Dataset(Xv, reference=dev, params={"device_binning": True}).construct()
    _same(hv.binned(), dv.binned())


def test_device_binning_several_chunks(lgb):
    X = _matrix(400000, 3, wide=True)  # 46 columns: 64 MB chunks of about 360k rows, two of them
    params = {"max_bin": 63, "categorical_feature": [5]}
    host = lgb.Dataset(X, params=params).construct().binned()
    for _ in range(2):
        dev = lgb.Dataset(X, params=dict(params, device_binning=True)).construct().binned()
        _same(host, dev)
