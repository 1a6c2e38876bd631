"""Metrics on the device (lgbm_b200_metric_eval) against the reference's
definitions (metric.rs:520-770): AUC bit for bit against the oracle's
sequential restatement (its sums are exact in FP64, so any order gives the
same value), the loss metrics within 1e-12 relative of a sequential NumPy
restatement (the device sums in another order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

K_EPS = float(np.float32(1e-15))
NEG_LOG_EPS = float(-np.log(np.float32(1e-15)))


@pytest.mark.parametrize("n", [1, 777, 100_000, 1_500_000])
def test_auc_matches_oracle(lgb, orc, n):
    rng = np.random.default_rng(n)
    label = (rng.random(n) < 0.3).astype(np.float32)
    score = rng.standard_normal(n)
    cases = [score, np.round(score, 1), np.where(rng.random(n) < 0.5, 0.0, -0.0)]  # distinct, tied, +/-0 ties
    for s in cases:
        assert lgb.metric("auc", label, s) == orc.auc(label, s)
    lab = label.copy()
    lab[rng.random(n) < 0.01] = np.nan  # a NaN label is neither class
    assert lgb.metric("auc", lab, score) == orc.auc(lab, score)
    assert lgb.metric("auc", np.ones(n, np.float32), score) == 1.0  # one class only


def _binary_ref(kind, label, score, sigmoid):
    with np.errstate(over="ignore"):  # exp(+large) = inf gives probability 0, as on the device
        prob = 1.0 / (1.0 + np.exp(-sigmoid * score))
    if kind == "binary_error":
        loss = np.where(prob <= 0.5, label > 0, label <= 0).astype(np.float64)
    else:
        neg = np.where(1.0 - prob > K_EPS, -np.log(np.maximum(1.0 - prob, 1e-300)), NEG_LOG_EPS)
        pos = np.where(prob > K_EPS, -np.log(np.maximum(prob, 1e-300)), NEG_LOG_EPS)
        loss = np.where(label <= 0, neg, pos)
    return float(np.sum(loss) / len(label))


def test_loss_metrics(lgb):
    rng = np.random.default_rng(7)
    n = 300_001
    yb = (rng.random(n) < 0.4).astype(np.float32)
    s = rng.standard_normal(n) * 4
    s[:10] = [60, -60, 40, -40, 0, 0.5, -0.5, 1e3, -1e3, 0]  # clamped probabilities included
    for kind in ("binary_logloss", "binary_error"):
        got = lgb.metric(kind, yb, s, sigmoid=1.5)
        assert got == pytest.approx(_binary_ref(kind, yb, s, 1.5), rel=1e-12, abs=0), kind
    yr = rng.standard_normal(n).astype(np.float32)
    l2 = float(np.sum((s - yr.astype(np.float64)) ** 2) / n)
    assert lgb.metric("l2", yr, s) == pytest.approx(l2, rel=1e-12)
    assert lgb.metric("rmse", yr, s) == pytest.approx(np.sqrt(l2), rel=1e-12)


def test_multiclass_metrics(lgb):
    rng = np.random.default_rng(8)
    n, k = 200_000, 5
    y = rng.integers(0, k, n).astype(np.float32)
    sc = rng.standard_normal((k, n)) * 2  # class-major
    z = sc - sc.max(axis=0)
    p = np.exp(z) / np.exp(z).sum(axis=0)
    pl = p[y.astype(int), np.arange(n)]
    ll = float(np.sum(np.where(pl > K_EPS, -np.log(pl), NEG_LOG_EPS)) / n)
    assert lgb.metric("multi_logloss", y, sc.ravel(), num_class=k) == pytest.approx(ll, rel=1e-12)
    for top_k in (1, 2):
        err = float(np.mean((p >= pl).sum(axis=0) > top_k))
        assert lgb.metric("multi_error", y, sc.ravel(), num_class=k, multi_error_top_k=top_k) == err


def test_ndcg_matches_oracle(lgb, orc):
    rng = np.random.default_rng(9)
    group = np.clip(rng.geometric(1.0 / 30.0, 3000), 1, 400).astype(np.int32)
    n = int(group.sum())
    label = rng.integers(0, 5, n).astype(np.float32)
    label[:group[0]] = 0  # a query whose best DCG is 0
    score = np.round(rng.standard_normal(n), 1)  # ties inside queries: the stable order decides
    for ks in ([1, 3, 5, 10], [10, 5, 1], [1000]):
        got = lgb.ndcg(label, score, group, ks)
        want = orc.ndcg(label, score, group, ks)
        assert np.array_equal(got, want), (ks, got, want)
