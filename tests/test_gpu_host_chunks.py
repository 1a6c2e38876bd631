"""The calls with host buffers that stream rows through the device in chunks
of 1M rows (the gradients of objectives with one value per row, and the
learner's score update), at sizes that take several chunks, one of them
partial."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


def test_gradients_several_chunks(lgb, orc):
    rng = np.random.default_rng(41)
    n = 2_600_000
    s = rng.standard_normal(n) * 3
    yb = (rng.random(n) < 0.4).astype(np.float32)
    for params, y in (({"objective": "binary"}, yb), ({"objective": "regression"}, rng.standard_normal(n))):
        p = lgb.resolve_params(params)
        for _ in range(2):  # the chunk streams are reused by the next call
            g, h = lgb.gradients(params, y, s)
            og, oh = orc.gradients(p, y, s)
            # exp is not correctly rounded on either side: allow one f32 ulp
            for a, o in ((g, og), (h, oh)):
                u = _ulps(a, o)
                assert u.max() <= 1, (params, u.max())
                assert np.mean(u == 0) > 0.99


@pytest.mark.parametrize("bagged", [False, True])
def test_add_leaf_outputs_several_chunks(lgb, bagged):
    rng = np.random.default_rng(42)
    n = 2_300_000
    X = rng.standard_normal((n, 6)).astype(np.float32)
    y = (X[:, 0] + 0.5 * X[:, 1] > 0).astype(np.float32)
    params = {"objective": "binary", "num_leaves": 31, "min_data_in_leaf": 20}
    ds = lgb.Dataset(X, y, params=params).construct()
    learner = lgb.Learner(ds, params)
    if bagged:  # rows out of the bag keep their scores
        learner.set_bagging(np.sort(rng.choice(n, int(0.7 * n), replace=False)).astype(np.uint32))
    g, h = lgb.gradients(params, y, np.zeros(n))
    tree = learner.train(g, h)[0]
    nl = int(tree["num_leaves"])
    beg, cnt, idx = learner.partition(0, nl)
    score = rng.standard_normal(n)
    for _ in range(2):
        lv = rng.standard_normal(nl)
        want = score.copy()
        for leaf in range(nl):
            rows = idx[beg[leaf]:beg[leaf] + cnt[leaf]]
            want[rows] += lv[leaf]
        learner.add_leaf_outputs(0, lv, score)
        assert np.array_equal(score, want)  # one FP64 add per row: bit-exact


def test_objective_handle_matches_stateless_gradients(lgb):
    """lgbm_b200_objective_* (labels bound once) gives exactly the gradients
    of lgbm_b200_gradients (labels passed every call): the same kernels."""
    rng = np.random.default_rng(43)
    n = 2_200_000
    cases = [({"objective": "binary"}, (rng.random(n) < 0.4).astype(np.float32), rng.standard_normal(n) * 3, None),
             ({"objective": "regression"}, rng.standard_normal(n).astype(np.float32), rng.standard_normal(n), None),
             ({"objective": "multiclass", "num_class": 3}, rng.integers(0, 3, 50000).astype(np.float32),
              rng.standard_normal(3 * 50000), None)]
    group = np.clip(rng.geometric(1.0 / 20.0, 2000), 1, 200).astype(np.int32)
    m = int(group.sum())
    cases.append(({"objective": "lambdarank"}, rng.integers(0, 5, m).astype(np.float32), rng.standard_normal(m),
                  group))
    for params, y, s, grp in cases:
        obj = lgb.Objective(params, y, group=grp)
        for _ in range(2):
            g, h = obj.gradients(s)
            g0, h0 = lgb.gradients(params, y, s, group=grp)
            assert np.array_equal(g, g0) and np.array_equal(h, h0), params["objective"]


def test_gradients_workspace_after_a_multiclass_call(lgb, orc):
    """The stateless gradient call keeps its device buffers between calls.
    A multiclass call on few rows (rows x classes values) followed by a
    binary call on more rows, but fewer values, must grow the label buffer:
    once the cache compared only the value count, and the second call's
    label copy overran the buffer ("invalid argument")."""
    rng = np.random.default_rng(43)
    n_mc, k, n_bin = 50_000, 10, 120_000
    ymc = rng.integers(0, k, n_mc).astype(np.float32)
    pmc = {"objective": "multiclass", "num_class": k}
    g, h = lgb.gradients(pmc, ymc, rng.standard_normal(n_mc * k))
    assert g.shape == (n_mc * k,) or g.size == n_mc * k
    yb = (rng.random(n_bin) < 0.3).astype(np.float32)
    s = rng.standard_normal(n_bin)
    pb = {"objective": "binary"}
    g, h = lgb.gradients(pb, yb, s)
    og, oh = orc.gradients(lgb.resolve_params(pb), yb, s)
    for a, o in ((g, og), (h, oh)):
        u = _ulps(np.asarray(a, np.float32).ravel(), np.asarray(o, np.float32).ravel())
        assert u.max() <= 1
        assert np.mean(u == 0) > 0.99
