"""ctypes wrapper of the CPU oracle (liblgbm_oracle.so).

TEST INFRASTRUCTURE ONLY: this is the checker the parity tests (and the
bench's CPU-baseline leg) run against the CUDA path. The product never
imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liblgbm_oracle.so")

i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
P = C.POINTER


class OracleParams(C.Structure):
    _fields_ = [("objective", i32), ("num_class", i32), ("sigmoid", f64), ("num_iterations", i32),
                ("learning_rate", f64), ("boost_from_average", i32), ("num_leaves", i32), ("max_depth", i32),
                ("min_data_in_leaf", i32), ("min_sum_hessian_in_leaf", f64), ("lambda_l1", f64), ("lambda_l2", f64),
                ("max_delta_step", f64), ("path_smooth", f64), ("min_gain_to_split", f64),
                ("max_cat_to_onehot", i32), ("max_cat_threshold", i32), ("cat_l2", f64), ("cat_smooth", f64),
                ("min_data_per_group", i32), ("bagging_fraction", f64), ("bagging_freq", i32),
                ("bagging_seed", i32), ("feature_fraction", f64), ("feature_fraction_seed", i32),
                ("use_quantized_grad", i32), ("num_grad_quant_bins", i32), ("stochastic_rounding", i32),
                ("quant_train_renew_leaf", i32), ("seed", i32), ("num_threads", i32), ("monotone_penalty", f64),
                ("lambdarank_truncation_level", i32), ("lambdarank_norm", i32)]


class OracleData(C.Structure):
    _fields_ = [("num_data", i64), ("num_features", i32), ("bins", P(C.c_uint8)), ("num_bin", P(i32)),
                ("missing_type", P(i32)), ("default_bin", P(i32)), ("most_freq_bin", P(i32)), ("bin_type", P(i32)),
                ("real_index", P(i32)), ("monotone", P(C.c_int8)), ("upper_bounds", P(f64)),
                ("ub_offsets", P(i64)), ("bin_to_cat", P(i32)), ("cat_offsets", P(i64))]


class OracleTreeView(C.Structure):
    _fields_ = [("num_leaves", i32), ("split_feature", P(i32)), ("split_feature_inner", P(i32)),
                ("split_gain", P(C.c_float)), ("threshold_in_bin", P(C.c_uint32)), ("threshold", P(f64)),
                ("decision_type", P(C.c_int8)), ("left_child", P(i32)), ("right_child", P(i32)),
                ("leaf_value", P(f64)), ("leaf_weight", P(f64)), ("leaf_count", P(i32)),
                ("internal_value", P(f64)), ("internal_weight", P(f64)), ("internal_count", P(i32)),
                ("leaf_depth", P(i32)), ("num_cat", i32), ("cat_boundaries", P(i32)),
                ("cat_threshold", P(C.c_uint32)), ("num_cat_threshold", i32), ("shrinkage", f64)]


class OracleFeature(C.Structure):
    _fields_ = [("num_bin", i32), ("missing_type", i32), ("default_bin", i32), ("most_freq_bin", i32),
                ("bin_type", i32), ("monotone_type", i32), ("offset", i32), ("penalty", f64), ("use_constraint", i32),
                ("constraint_min", f64), ("constraint_max", f64)]


class OracleSplit(C.Structure):
    _fields_ = [("splittable", i32), ("threshold", C.c_uint32), ("gain", f64), ("left_output", f64),
                ("right_output", f64), ("left_count", i32), ("right_count", i32), ("left_sum_gradient", f64),
                ("left_sum_hessian", f64), ("right_sum_gradient", f64), ("right_sum_hessian", f64),
                ("default_left", i32), ("num_cat", i32), ("cat_threshold", C.c_uint32 * 256),
                ("left_sum_gh", i64), ("right_sum_gh", i64)]


class OracleBinParams(C.Structure):
    _fields_ = [("max_bin", i32), ("min_data_in_bin", i32), ("min_data_in_leaf", i32),
                ("bin_construct_sample_cnt", i32), ("data_random_seed", i32), ("use_missing", i32),
                ("zero_as_missing", i32), ("feature_pre_filter", i32), ("categorical", P(i32)),
                ("num_categorical", i32)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_train.argtypes = [P(OracleParams), P(OracleData), P(C.c_float), P(i32), i32, P(OracleData),
                                   P(C.c_void_p)]
        L.oracle_booster_free.argtypes = [C.c_void_p]
        L.oracle_booster_update.argtypes = [C.c_void_p, P(i32)]
        L.oracle_train_tree.argtypes = [P(OracleParams), P(OracleData), P(C.c_float), P(C.c_float),
                                        P(C.c_uint32), i64, i32, P(C.c_uint8), P(C.c_void_p)]
        L.oracle_booster_partition.argtypes = [C.c_void_p, P(i32), P(i32), P(C.c_uint32)]
        L.oracle_booster_num_trees.argtypes = [C.c_void_p]
        L.oracle_booster_tree.argtypes = [C.c_void_p, i32, P(OracleTreeView)]
        L.oracle_booster_trace.argtypes = [C.c_void_p, i32, P(i32), P(i32), P(i32), P(C.c_uint32), P(f64)]
        L.oracle_booster_scores.argtypes = [C.c_void_p, C.c_int, P(f64)]
        L.oracle_predict_raw.argtypes = [C.c_void_p, P(C.c_float), i64, i32, P(f64)]
        L.oracle_auc.restype = f64
        L.oracle_auc.argtypes = [P(C.c_float), P(f64), i64]
        L.oracle_ndcg.argtypes = [P(C.c_float), P(f64), P(i32), i32, P(i32), i32, P(f64)]
        L.oracle_gradients.argtypes = [i32, i32, f64, P(C.c_float), P(f64), i64, P(i32), i32, i32, i32,
                                       P(C.c_float), P(C.c_float)]
        L.oracle_hist.argtypes = [P(OracleData), P(C.c_uint32), i64, P(C.c_float), P(C.c_float), P(i64), P(f64),
                                  P(i64)]
        L.oracle_find_best_threshold.argtypes = [P(OracleFeature), P(OracleParams), P(f64), P(i64), f64, f64, i64,
                                                 f64, f64, i32, f64, P(OracleSplit)]
        L.oracle_discretize.argtypes = [i32, i32, i32, i32, i64, i32, i32, P(C.c_float), P(C.c_float), P(i64),
                                        P(f64)]
        L.oracle_mt19937.argtypes = [C.c_uint32, i32, P(C.c_uint32)]
        L.oracle_lcg_sample.argtypes = [i32, i32, i32, P(i32), P(i32)]
        L.oracle_block_info.argtypes = [i64, i64, i64, P(i64)]
        L.oracle_dataset_create.argtypes = [P(C.c_float), i64, i32, P(OracleBinParams), P(C.c_void_p)]
        L.oracle_dataset_create_valid.argtypes = [P(C.c_float), i64, i32, C.c_void_p, P(C.c_void_p)]
        L.oracle_dataset_view.argtypes = [C.c_void_p, P(OracleData), P(i32)]
        L.oracle_dataset_feature_infos.restype = C.c_char_p
        L.oracle_dataset_feature_infos.argtypes = [C.c_void_p]
        L.oracle_dataset_free.argtypes = [C.c_void_p]
        L.oracle_model_to_string.argtypes = [C.c_void_p, i32, C.c_char_p, P(C.c_int8), i32, P(C.c_char_p)]
        L.oracle_fix_hist.argtypes = [i32, i32, i32, f64, f64, P(f64)]
        L.oracle_better_than.restype = i32
        L.oracle_better_than.argtypes = [f64, i32, f64, i32]
        L.oracle_to_i8.restype = C.c_int8
        L.oracle_to_i8.argtypes = [f64]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().oracle_last_error().decode())


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(P(ct))


OBJ = {"binary": 0, "regression": 1, "regression_l2": 1, "l2": 1, "mse": 1, "multiclass": 2, "softmax": 2,
       "lambdarank": 3}


def params_struct(p, num_iterations=1):
    """OracleParams from a resolved parameter dict (lgbm_b200.resolve_params)."""
    return OracleParams(
        OBJ[p["objective"]], int(p["num_class"]), float(p["sigmoid"]), int(num_iterations), float(p["learning_rate"]),
        int(bool(p["boost_from_average"])), int(p["num_leaves"]), int(p["max_depth"]), int(p["min_data_in_leaf"]),
        float(p["min_sum_hessian_in_leaf"]), float(p["lambda_l1"]), float(p["lambda_l2"]), float(p["max_delta_step"]),
        float(p["path_smooth"]), float(p["min_gain_to_split"]), int(p["max_cat_to_onehot"]),
        int(p["max_cat_threshold"]), float(p["cat_l2"]), float(p["cat_smooth"]), int(p["min_data_per_group"]),
        float(p["bagging_fraction"]), int(p["bagging_freq"]), int(p["bagging_seed"]), float(p["feature_fraction"]),
        int(p["feature_fraction_seed"]), int(p["hist_precision"] == "quantized"), int(p["num_grad_quant_bins"]),
        int(bool(p["stochastic_rounding"])), int(bool(p["quant_train_renew_leaf"])), int(p["seed"]),
        int(p["num_threads"]) if p["num_threads"] else 1, float(p["monotone_penalty"]),
        int(p["lambdarank_truncation_level"]), int(bool(p["lambdarank_norm"])))


class Data:
    """OracleData over a binned dict (lgbm_b200.Dataset.binned()); keeps the arrays alive."""

    def __init__(self, b, monotone=None):
        self.b = b
        self.bins = np.ascontiguousarray(b["bins"], dtype=np.uint8)
        self.keep = [self.bins]
        d = OracleData()
        d.num_data = int(b["num_data"])
        d.num_features = int(b["num_features"])
        d.bins = _p(self.bins, C.c_uint8)
        for name in ("num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index"):
            a = np.ascontiguousarray(b[name], dtype=np.int32)
            self.keep.append(a)
            setattr(d, name, _p(a, i32))
        if monotone is not None:
            m = np.ascontiguousarray([monotone[int(r)] if int(r) < len(monotone) else 0 for r in b["real_index"]],
                                     dtype=np.int8)
            self.keep.append(m)
            d.monotone = _p(m, C.c_int8)
        for name, ct, dt in (("upper_bounds", f64, np.float64), ("ub_offsets", i64, np.int64),
                             ("bin_to_cat", i32, np.int32), ("cat_offsets", i64, np.int64)):
            a = np.ascontiguousarray(b[name], dtype=dt)
            if a.size == 0:
                a = np.zeros(1, dt)
            self.keep.append(a)
            setattr(d, name, _p(a, ct))
        self.s = d


def _tree(v):
    nl = v.num_leaves
    nn = nl - 1

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n > 0 else np.zeros(0, dt)

    t = {"num_leaves": nl}
    for name, n, dt in (("split_feature", nn, np.int32), ("split_feature_inner", nn, np.int32),
                        ("split_gain", nn, np.float32), ("threshold_in_bin", nn, np.uint32),
                        ("threshold", nn, np.float64), ("decision_type", nn, np.int8), ("left_child", nn, np.int32),
                        ("right_child", nn, np.int32), ("leaf_value", nl, np.float64), ("leaf_weight", nl, np.float64),
                        ("leaf_count", nl, np.int32), ("internal_value", nn, np.float64),
                        ("internal_weight", nn, np.float64), ("internal_count", nn, np.int32),
                        ("leaf_depth", nl, np.int32)):
        t[name] = arr(getattr(v, name), n, dt)
    t["num_cat"] = v.num_cat
    t["cat_boundaries"] = arr(v.cat_boundaries, v.num_cat + 1, np.int32)
    t["cat_threshold"] = arr(v.cat_threshold, v.num_cat_threshold, np.uint32)
    t["shrinkage"] = v.shrinkage
    return t


class Model:
    def __init__(self, h, ntpi, n, nv):
        self.h = h
        self.ntpi = ntpi
        self.n = n
        self.nv = nv
        L = lib()
        self.trees = []
        for i in range(L.oracle_booster_num_trees(h)):
            v = OracleTreeView()
            _check(L.oracle_booster_tree(h, i, C.byref(v)))
            self.trees.append(_tree(v))

    def trace(self, i):
        L = lib()
        n = i32()
        _check(L.oracle_booster_trace(self.h, i, C.byref(n), None, None, None, None))
        leaf = np.zeros(n.value, np.int32)
        feat = np.zeros(n.value, np.int32)
        thr = np.zeros(n.value, np.uint32)
        gain = np.zeros(n.value, np.float64)
        _check(L.oracle_booster_trace(self.h, i, C.byref(n), _p(leaf, i32), _p(feat, i32), _p(thr, C.c_uint32),
                                      _p(gain, f64)))
        return leaf, feat, thr, gain

    def scores(self, valid=False):
        n = self.nv if valid else self.n
        out = np.zeros(n * self.ntpi, np.float64)
        _check(lib().oracle_booster_scores(self.h, int(valid), _p(out, f64)))
        return out.reshape(self.ntpi, n)

    def predict_raw(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(X.shape[0] * self.ntpi, np.float64)
        _check(lib().oracle_predict_raw(self.h, _p(X, C.c_float), X.shape[0], X.shape[1], _p(out, f64)))
        return out.reshape(X.shape[0], self.ntpi)

    def update(self):
        """One more boosting iteration (Gbdt::train_one_iter); True when training stopped."""
        stop = i32()
        _check(lib().oracle_booster_update(self.h, C.byref(stop)))
        L = lib()
        for i in range(len(self.trees), L.oracle_booster_num_trees(self.h)):
            v = OracleTreeView()
            _check(L.oracle_booster_tree(self.h, i, C.byref(v)))
            self.trees.append(_tree(v))
        return bool(stop.value)

    def model_to_string(self, num_total_features, feature_infos, monotone=None):
        """Gbdt::save_model_to_string (io.rs:13-85) up to the feature importances."""
        out = C.c_char_p()
        mono = None if monotone is None else np.ascontiguousarray(monotone, dtype=np.int8)
        _check(lib().oracle_model_to_string(self.h, int(num_total_features), " ".join(feature_infos).encode(),
                                            _p(mono, C.c_int8), 0 if mono is None else len(mono), C.byref(out)))
        return out.value.decode()

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.oracle_booster_free(self.h)
            self.h = None


def train(p, binned, label, num_iterations, valid_binned=None, group=None, monotone=None):
    """The reference's boosting loop on the CPU (one thread)."""
    d = Data(binned, monotone)
    vd = Data(valid_binned) if valid_binned is not None else None
    label = np.ascontiguousarray(label, dtype=np.float32)
    bnd = None
    nq = 0
    if group is not None:
        bnd = np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
        nq = len(group)
    ps = params_struct(p, num_iterations)
    h = C.c_void_p()
    _check(lib().oracle_train(C.byref(ps), C.byref(d.s), _p(label, C.c_float), _p(bnd, i32), nq,
                              C.byref(vd.s) if vd else None, C.byref(h)))
    ntpi = int(p["num_class"]) if OBJ[p["objective"]] == 2 else 1
    m = Model(h, ntpi, int(binned["num_data"]), int(valid_binned["num_data"]) if valid_binned else 0)
    # the booster keeps pointers into the binned arrays: they live as long as the model
    m.data, m.vdata = d, vd
    return m


def train_trees(p, binned, grad, hess, num_trees=1, bag=None, bytree=None, monotone=None):
    """SerialTreeLearner::train on given (class-major) gradients: `num_trees`
    trees in sequence on one learner. Returns the Model (trees unshrunk)."""
    d = Data(binned, monotone)
    ps = params_struct(p, 1)
    g = np.ascontiguousarray(grad, np.float32)
    h = np.ascontiguousarray(hess, np.float32)
    bg = None if bag is None else np.ascontiguousarray(bag, np.uint32)
    bt = None if bytree is None else np.ascontiguousarray(bytree, np.uint8)
    out = C.c_void_p()
    _check(lib().oracle_train_tree(C.byref(ps), C.byref(d.s), _p(g, C.c_float), _p(h, C.c_float),
                                   _p(bg, C.c_uint32), 0 if bg is None else len(bg), num_trees, _p(bt, C.c_uint8),
                                   C.byref(out)))
    m = Model(out, 1, int(binned["num_data"]), 0)
    m.data = d
    return m


def partition(model, num_leaves, n):
    beg = np.zeros(num_leaves, np.int32)
    cnt = np.zeros(num_leaves, np.int32)
    idx = np.zeros(n, np.uint32)
    _check(lib().oracle_booster_partition(model.h, _p(beg, i32), _p(cnt, i32), _p(idx, C.c_uint32)))
    return beg, cnt, idx


def gradients(p, label, scores, group=None):
    label = np.ascontiguousarray(label, dtype=np.float32)
    scores = np.ascontiguousarray(scores, dtype=np.float64)
    g = np.zeros(scores.shape, np.float32)
    h = np.zeros(scores.shape, np.float32)
    bnd = None
    nq = 0
    if group is not None:
        bnd = np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
        nq = len(group)
    _check(lib().oracle_gradients(OBJ[p["objective"]], int(p["num_class"]), float(p["sigmoid"]),
                                  _p(label, C.c_float), _p(scores, f64), len(label), _p(bnd, i32), nq,
                                  int(p["lambdarank_truncation_level"]), int(bool(p["lambdarank_norm"])),
                                  _p(g, C.c_float), _p(h, C.c_float)))
    return g, h


def hist(binned, rows, g, h):
    d = Data(binned)
    g = np.ascontiguousarray(g, dtype=np.float32)
    h = np.ascontiguousarray(h, dtype=np.float32)
    total = int(np.sum(binned["num_bin"] - (binned["most_freq_bin"] == 0)))
    out = np.zeros(2 * total, np.float64)
    r = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
    _check(lib().oracle_hist(C.byref(d.s), _p(r, C.c_uint32), 0 if r is None else len(r), _p(g, C.c_float),
                             _p(h, C.c_float), None, _p(out, f64), None))
    return out


def auc(label, score):
    label = np.ascontiguousarray(label, dtype=np.float32)
    score = np.ascontiguousarray(score, dtype=np.float64)
    return lib().oracle_auc(_p(label, C.c_float), _p(score, f64), len(label))


def ndcg(label, score, group, ks):
    label = np.ascontiguousarray(label, dtype=np.float32)
    score = np.ascontiguousarray(score, dtype=np.float64)
    bnd = np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
    ks = np.ascontiguousarray(ks, dtype=np.int32)
    out = np.zeros(len(ks), np.float64)
    _check(lib().oracle_ndcg(_p(label, C.c_float), _p(score, f64), _p(bnd, i32), len(group), _p(ks, i32), len(ks),
                             _p(out, f64)))
    return out


class Dataset:
    """The oracle's own binning of a dense f32 matrix (Dataset::from_dense,
    dataset.rs:355; binning.cpp). `binned()` has the layout of the product's
    Dataset.binned(); `feature_infos` is Dataset::feature_infos (dataset.rs:770)."""

    def __init__(self, X, params, categorical=None, reference=None):
        X = np.ascontiguousarray(X, dtype=np.float32)
        n, ncol = X.shape
        h = C.c_void_p()
        if reference is not None:
            _check(lib().oracle_dataset_create_valid(_p(X, C.c_float), n, ncol, reference.h, C.byref(h)))
        else:
            cats = np.ascontiguousarray(sorted(set(categorical or [])), dtype=np.int32)
            bp = OracleBinParams(int(params["max_bin"]), int(params["min_data_in_bin"]),
                                 int(params["min_data_in_leaf"]), int(params["bin_construct_sample_cnt"]),
                                 int(params["data_random_seed"]), int(bool(params["use_missing"])),
                                 int(bool(params["zero_as_missing"])), int(bool(params["feature_pre_filter"])),
                                 _p(cats, i32) if len(cats) else None, len(cats))
            _check(lib().oracle_dataset_create(_p(X, C.c_float), n, ncol, C.byref(bp), C.byref(h)))
        self.h = h
        v = OracleData()
        nt = i32()
        _check(lib().oracle_dataset_view(h, C.byref(v), C.byref(nt)))
        nf = v.num_features
        nd = int(v.num_data)
        b = {"num_data": nd, "num_features": nf, "num_total_features": int(nt.value),
             "bins": np.ctypeslib.as_array(v.bins, shape=(nd * nf,)).reshape(nd, nf).copy()
             if nf else np.zeros((nd, 0), np.uint8)}
        for name in ("num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index"):
            b[name] = np.ctypeslib.as_array(getattr(v, name), shape=(nf,)).copy() if nf else np.zeros(0, np.int32)
        b["ub_offsets"] = np.ctypeslib.as_array(v.ub_offsets, shape=(nf + 1,)).copy()
        b["cat_offsets"] = np.ctypeslib.as_array(v.cat_offsets, shape=(nf + 1,)).copy()
        nu, nc = int(b["ub_offsets"][-1]), int(b["cat_offsets"][-1])
        b["upper_bounds"] = np.ctypeslib.as_array(v.upper_bounds, shape=(nu,)).copy() if nu else np.zeros(0)
        b["bin_to_cat"] = (np.ctypeslib.as_array(v.bin_to_cat, shape=(nc,)).copy() if nc
                           else np.zeros(0, np.int32))
        self._binned = b
        self.feature_infos = lib().oracle_dataset_feature_infos(h).decode().split(" ")

    def binned(self):
        return self._binned

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.oracle_dataset_free(self.h)
            self.h = None
