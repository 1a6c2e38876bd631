"""The reference's known-answer tests that reach the device, through the C ABI:

- bin.rs:762-788: the histogram of a row subset with ordered gradients equals
  the dense reference sums (exact: every sum here is exact in FP64);
- split.rs:1476-1484 (tie_break_prefers_smaller_feature) on the device: two
  identical columns give every candidate split the same gain twice, and the
  device picks the one of the smaller feature index every time.
"""
import numpy as np
import pytest

from test_oracle_kat import bin_rs_histogram_case

pytestmark = pytest.mark.gpu


class _Binned:
    """A dataset given by its binned dict (what Learner reads)."""

    def __init__(self, b):
        self.b = b

    def construct(self, params=None):
        return self

    def binned(self):
        return self.b


def test_bin_histogram_on_the_device(lgb):
    b, g, rows, want = bin_rs_histogram_case()
    learner = lgb.Learner(_Binned(b), {"objective": "regression", "min_data_in_leaf": 1})
    learner.train(g, g)  # loads the gradients
    got = learner.histogram(rows)
    assert list(got) == list(want)


@pytest.mark.parametrize("form", ["f64", "quantized"])
def test_tie_break_prefers_smaller_feature_on_the_device(lgb, orc, form):
    rng = np.random.default_rng(17)
    n = 20000
    base = rng.standard_normal((n, 4)).astype(np.float32)
    # column 3 repeats column 1: each of its candidates ties with column 1's
    X = np.concatenate([base, base[:, 1:2]], axis=1)
    y = (base[:, 0] + base[:, 1] - 0.5 * base[:, 2] + 0.3 * rng.standard_normal(n) > 0).astype(np.float32)
    params = {"objective": "binary", "num_leaves": 31, "hist_precision": form, "num_threads": 8}
    ds = lgb.Dataset(X, y, params=params)
    p = lgb.resolve_params(params)
    g, h = orc.gradients(p, y, np.zeros(n))
    t = lgb.Learner(ds, params).train(g, h)[0]
    assert 1 in set(t["split_feature"])
    assert 4 not in set(t["split_feature"])  # the duplicate never wins a tie
