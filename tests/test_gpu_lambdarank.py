"""Lambdarank gradients on the device against the oracle's restatement of
LambdarankNDCG::one_query (objective/rank.rs:192-262).

Without the normalisation every value is a sequence of f32 additions in the
reference's pair order, so the device must match bit for bit. With it, the
FP64 sum of the lambdas is also formed in the reference's order, and the
factor log2(1 + s) / s uses CUDA's log2 (within 1 ulp of the host's), so the
values match within 1 ulp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _queries(seed):
    rng = np.random.default_rng(seed)
    # sizes around the lane and pass boundaries (32 rows per warp pass, 30 outer positions)
    group = np.concatenate([[1, 2, 29, 30, 31, 32, 33, 63, 64, 65, 500, 1000],
                            np.clip(rng.geometric(1.0 / 40.0, 600), 1, 300)]).astype(np.int32)
    rng.shuffle(group)
    n = int(group.sum())
    label = rng.integers(0, 5, n).astype(np.float32)
    score = np.round(rng.standard_normal(n), 1)  # ties: the stable order decides
    score[rng.random(n) < 0.01] = -np.inf  # the minimum score: its pairs are skipped
    return group, label, score


def _ulps(a, b):
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


@pytest.mark.parametrize("trunc", [1, 5, 30, 1000])
def test_unnormalised_gradients_bit_exact(lgb, orc, trunc):
    group, label, score = _queries(trunc)
    params = {"objective": "lambdarank", "lambdarank_norm": False, "lambdarank_truncation_level": trunc}
    g, h = lgb.gradients(params, label, score, group=group)
    og, oh = orc.gradients(lgb.resolve_params(params), label, score, group)
    assert np.array_equal(g, og) and np.array_equal(h, oh)


def test_normalised_gradients_within_one_ulp(lgb, orc):
    group, label, score = _queries(7)
    params = {"objective": "lambdarank"}
    g, h = lgb.gradients(params, label, score, group=group)
    og, oh = orc.gradients(lgb.resolve_params(params), label, score, group)
    assert _ulps(g, og).max() <= 1 and _ulps(h, oh).max() <= 1
    assert np.mean(_ulps(g, og) == 0) > 0.9
    # the objective handle (labels bound once) runs the same kernels
    obj = lgb.Objective(params, label, group=group)
    g2, h2 = obj.gradients(score)
    assert np.array_equal(g2, g) and np.array_equal(h2, h)
