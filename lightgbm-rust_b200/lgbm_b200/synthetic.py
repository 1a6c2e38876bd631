"""Seeded synthetic workloads with the shapes, sizes and value distributions of
the five benchmark configurations (no public dataset is involved; the
"HIGGS-like" 28-feature shape follows the reference bench's description).

`make(cfg, scale)` returns a dict with X / y (and held-out X_valid / y_valid,
query sizes `group`, `categorical`), the training parameters and the round
count. `scale` < 1 shrinks the row count (and query count) for tests.
"""
import numpy as np


def _label_c0(X, rng):
    """Bernoulli(sigmoid(x0 + x1*x2 - 0.5*x3^2 + 0.3*eps))."""
    z = X[:, 0] + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2 + 0.3 * rng.standard_normal(X.shape[0])
    p = 1.0 / (1.0 + np.exp(-z))
    return (rng.random(X.shape[0]) < p).astype(np.float32)


def config0(scale=1.0, seed=0):
    """Binary, 20,000 train + 5,000 held-out x 28 N(0,1); 31 leaves, 100 rounds."""
    rng = np.random.default_rng(seed)
    n, nv = max(200, int(20000 * scale)), max(50, int(5000 * scale))
    X = rng.standard_normal((n + nv, 28), dtype=np.float32)
    y = _label_c0(X, rng)
    params = dict(objective="binary", max_bin=255, num_leaves=31, learning_rate=0.1, min_data_in_leaf=20)
    return dict(X=X[:n], y=y[:n], X_valid=X[n:], y_valid=y[n:], params=params, num_rounds=100,
                name="binary 20k+5k x 28, 31 leaves")


def config1(scale=1.0, seed=1):
    """L2 regression, 1,000,000 x 100 (60 N(0,1), 30 lognormal, 10 integer U{0..15}), 5% NaN."""
    rng = np.random.default_rng(seed)
    n = max(1000, int(1_000_000 * scale))
    X = np.empty((n, 100), np.float32)
    X[:, :60] = rng.standard_normal((n, 60), dtype=np.float32)
    X[:, 60:90] = rng.lognormal(0.0, 1.0, (n, 30)).astype(np.float32)
    X[:, 90:] = rng.integers(0, 16, (n, 10)).astype(np.float32)
    y = np.sin(np.nan_to_num(X[:, 0])).astype(np.float64)
    for _ in range(10):  # axis-aligned stumps
        j = int(rng.integers(0, 100))
        t = float(np.quantile(X[: min(n, 100000), j], rng.uniform(0.1, 0.9)))
        y += rng.normal(0.0, 1.0) * (X[:, j] > t)
    y += rng.normal(0.0, 0.1, n)
    X[rng.random((n, 100)) < 0.05] = np.nan  # MCAR
    params = dict(objective="regression", max_bin=255, num_leaves=255, learning_rate=0.05, bagging_fraction=0.8,
                  bagging_freq=1, feature_fraction=0.8)
    return dict(X=X, y=y.astype(np.float32), params=params, num_rounds=500,
                name="L2 1M x 100, 5% NaN, 255 leaves, bagging 0.8, feature_fraction 0.8")


def config2(scale=1.0, seed=2):
    """Binary, 10,000,000 train + 1,000,000 held-out x 28 (21 N(0,1) + 7 heavy-tailed)."""
    rng = np.random.default_rng(seed)
    n, nv = max(1000, int(10_000_000 * scale)), max(100, int(1_000_000 * scale))
    N = n + nv
    X = np.empty((N, 28), np.float32)
    X[:, :21] = rng.standard_normal((N, 21), dtype=np.float32)
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7), (8, 9), (10, 11), (12, 13)]
    for k, (a, b) in enumerate(pairs):
        if k % 2 == 0:
            X[:, 21 + k] = X[:, a] * X[:, b]
        else:
            X[:, 21 + k] = X[:, a] / (np.abs(X[:, b]) + np.float32(0.1))
    y = _label_c0(X, rng)
    params = dict(objective="binary", max_bin=255, num_leaves=255, learning_rate=0.1)
    return dict(X=X[:n], y=y[:n], X_valid=X[n:], y_valid=y[n:], params=params, num_rounds=500,
                name="binary 10M+1M x 28, 255 leaves")


def config3(scale=1.0, seed=3):
    """Multiclass K=10, 2,000,000 x 200 (180 N(0,1) + 20 categorical Zipf(1.2) over 50 categories)."""
    rng = np.random.default_rng(seed)
    n = max(2000, int(2_000_000 * scale))
    X = np.empty((n, 200), np.float32)
    X[:, :180] = rng.standard_normal((n, 180), dtype=np.float32)
    p = 1.0 / np.arange(1, 51) ** 1.2
    p /= p.sum()
    cats = rng.choice(50, size=(n, 20), p=p)
    X[:, 180:] = cats.astype(np.float32)
    W = rng.standard_normal((180, 10)) / np.sqrt(180.0)
    E = rng.standard_normal((20, 50, 10)) * 0.3
    score = X[:, :180].astype(np.float64) @ W
    for j in range(20):
        score += E[j][cats[:, j]]
    score += rng.gumbel(size=(n, 10))
    y = np.argmax(score, axis=1).astype(np.float32)
    params = dict(objective="multiclass", num_class=10, num_leaves=127, max_cat_to_onehot=4,
                  categorical_feature=list(range(180, 200)))
    return dict(X=X, y=y, params=params, num_rounds=300, categorical=list(range(180, 200)),
                name="multiclass K=10, 2M x 200 (20 categorical)")


def config4(scale=1.0, seed=4):
    """LambdaRank, 500,000 queries (geometric sizes, mean 40, in [1, 1000]) x 136."""
    rng = np.random.default_rng(seed)
    nq = max(50, int(500_000 * scale))
    group = np.clip(rng.geometric(1.0 / 40.0, nq), 1, 1000).astype(np.int32)
    n = int(group.sum())
    X = np.empty((n, 136), np.float32)
    X[:, :68] = rng.standard_normal((n, 68), dtype=np.float32)
    X[:, 68:] = rng.random((n, 68), dtype=np.float32)
    X[rng.random((n, 136)) < 0.2] = 0.0
    w = rng.standard_normal(136) / np.sqrt(136.0)
    s = X.astype(np.float64) @ w + 0.5 * rng.standard_normal(n)
    qs = np.quantile(s, [0.5, 0.75, 0.9, 0.97])
    y = np.searchsorted(qs, s).astype(np.float32)  # relevance 0..4
    params = dict(objective="lambdarank", num_leaves=255, eval_at=[1, 3, 5, 10])
    return dict(X=X, y=y, group=group, params=params, num_rounds=300,
                name="lambdarank 500k queries (~20M rows) x 136")


CONFIGS = [config0, config1, config2, config3, config4]


def make(cfg, scale=1.0, seed=None):
    f = CONFIGS[cfg]
    return f(scale) if seed is None else f(scale, seed)
