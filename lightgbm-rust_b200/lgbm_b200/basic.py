"""Dataset / Booster / train over liblgbm_b200, mirroring the names and
argument meaning of lightgbm-rust's Python API (python/lightgbm_rust/basic.py
Dataset :710, Booster :1364, engine.py train :50) for the tree-learning path.

Binning stays on the host (Dataset); the bin matrix is uploaded once to the
GPU learner, and every boosting iteration runs on the device.
"""
import ctypes as C

import numpy as np

from . import _lib as L
from . import model_text

# config.rs:517-602 defaults for the parameters this path reads
DEFAULTS = {
    "objective": "regression", "num_class": 1, "sigmoid": 1.0, "learning_rate": 0.1, "num_leaves": 31,
    "max_depth": -1, "min_data_in_leaf": 20, "min_sum_hessian_in_leaf": 1e-3, "lambda_l1": 0.0, "lambda_l2": 0.0,
    "max_delta_step": 0.0, "path_smooth": 0.0, "min_gain_to_split": 0.0, "max_cat_to_onehot": 4,
    "max_cat_threshold": 32, "cat_l2": 10.0, "cat_smooth": 10.0, "min_data_per_group": 100,
    "monotone_penalty": 0.0, "max_bin": 255, "min_data_in_bin": 3, "bin_construct_sample_cnt": 200000,
    "data_random_seed": 1, "bagging_seed": 3, "feature_fraction_seed": 2, "objective_seed": 5, "extra_seed": 6,
    "bagging_fraction": 1.0, "bagging_freq": 0, "feature_fraction": 1.0, "use_quantized_grad": False,
    "num_grad_quant_bins": 4, "quant_train_renew_leaf": False, "stochastic_rounding": True, "use_missing": True,
    "zero_as_missing": False, "feature_pre_filter": True, "boost_from_average": True, "seed": 0,
    "lambdarank_truncation_level": 30, "lambdarank_norm": True, "num_threads": 0, "monotone_constraints": None,
    "categorical_feature": None,
    # B200 path knobs
    "hist_precision": "f64", "device": 0, "use_cuda_graph": True, "hist_rows_per_block": 0, "persistent_grow": False,
    "device_binning": False,
}

ALIASES = {
    "num_iterations": "num_boost_round", "num_iteration": "num_boost_round", "n_estimators": "num_boost_round",
    "num_round": "num_boost_round", "eta": "learning_rate", "shrinkage_rate": "learning_rate",
    "num_leaf": "num_leaves", "max_leaves": "num_leaves", "min_data": "min_data_in_leaf",
    "min_child_samples": "min_data_in_leaf", "min_child_weight": "min_sum_hessian_in_leaf",
    "reg_alpha": "lambda_l1", "reg_lambda": "lambda_l2", "lambda": "lambda_l2",
    "sub_feature": "feature_fraction", "colsample_bytree": "feature_fraction", "sub_row": "bagging_fraction",
    "subsample": "bagging_fraction", "bagging": "bagging_fraction", "subsample_freq": "bagging_freq",
    "min_split_gain": "min_gain_to_split", "random_state": "seed", "random_seed": "seed",
    "num_classes": "num_class", "application": "objective", "app": "objective",
}

OBJECTIVES = {"binary": L.OBJ_BINARY, "regression": L.OBJ_REGRESSION, "regression_l2": L.OBJ_REGRESSION,
              "l2": L.OBJ_REGRESSION, "mse": L.OBJ_REGRESSION, "multiclass": L.OBJ_MULTICLASS,
              "softmax": L.OBJ_MULTICLASS, "lambdarank": L.OBJ_LAMBDARANK}
HIST = {"f64": L.HIST_F64, "f32c": L.HIST_F32C, "quantized": L.HIST_QUANT}


def resolve_params(params):
    """Defaults, aliases and the seed derivation of config.rs:796-806."""
    p = dict(DEFAULTS)
    user = {}
    for k, v in (params or {}).items():
        user[ALIASES.get(k, k)] = v
    p.update(user)
    if "seed" in user and user["seed"] is not None:
        x = int(user["seed"]) & 0xFFFFFFFF

        def next_short():
            nonlocal x
            x = (x * 214013 + 2531011) & 0xFFFFFFFF
            return ((x >> 16) & 0x7FFF) % 32767

        for name in ("data_random_seed", "bagging_seed", "drop_seed", "feature_fraction_seed", "objective_seed",
                     "extra_seed"):
            v = next_short()
            if name not in user:
                p[name] = v
    if p.get("use_quantized_grad"):
        p["hist_precision"] = "quantized"
    if p["objective"] not in OBJECTIVES:
        raise L.LightGBMError(L.ERR_UNSUPPORTED, f"objective {p['objective']!r} is not on the B200 path")
    return p


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Dataset:
    """Binned training / validation data (python/lightgbm_rust/basic.py:710)."""

    def __init__(self, data, label=None, group=None, categorical_feature=None, params=None, reference=None):
        self.data = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
        if self.data.ndim != 2:
            raise L.LightGBMError(L.ERR_INVALID_DATA, "data must be 2-D")
        self.label = None if label is None else np.ascontiguousarray(np.asarray(label, dtype=np.float32))
        self.group = None if group is None else np.asarray(group, dtype=np.int32)
        self.categorical_feature = list(categorical_feature or [])
        self.params = dict(params or {})
        self.reference = reference
        self._handle = None
        self._view = None

    def construct(self, params=None):
        if self._handle is not None:
            return self
        p = resolve_params({**(params or {}), **self.params})
        lib = L.lib()
        n, ncol = self.data.shape
        h = C.c_void_p()
        # device_binning: the rows are binned on the CUDA device `device` (the
        # same dataset, byte for byte; the mappers still come from the host)
        dev = int(p["device"]) if p.get("device_binning") else -1
        if self.reference is not None:
            self.reference.construct(params)
            if dev >= 0:
                L.check(lib.lgbm_b200_dataset_create_valid_device(_ptr(self.data, C.c_float), n, ncol,
                                                                  self.reference._handle, dev, C.byref(h)))
            else:
                L.check(lib.lgbm_b200_dataset_create_valid(_ptr(self.data, C.c_float), n, ncol,
                                                           self.reference._handle, C.byref(h)))
        else:
            cats = np.asarray(self.categorical_feature or p.get("categorical_feature") or [], dtype=np.int32)
            bp = L.BinParams(int(p["max_bin"]), int(p["min_data_in_bin"]), int(p["min_data_in_leaf"]),
                             int(p["bin_construct_sample_cnt"]), int(p["data_random_seed"]), int(p["use_missing"]),
                             int(p["zero_as_missing"]), int(p["feature_pre_filter"]),
                             _ptr(cats, C.c_int32) if len(cats) else None, len(cats))
            self._cats = cats
            if dev >= 0:
                L.check(lib.lgbm_b200_dataset_create_device(_ptr(self.data, C.c_float), n, ncol, C.byref(bp), dev,
                                                            C.byref(h)))
            else:
                L.check(lib.lgbm_b200_dataset_create(_ptr(self.data, C.c_float), n, ncol, C.byref(bp), C.byref(h)))
        self._handle = h
        v = L.DatasetView()
        L.check(lib.lgbm_b200_dataset_view(h, C.byref(v)))
        self._view = v
        return self

    # numpy copies of the binned view
    def binned(self):
        self.construct()
        v = self._view
        nf = v.num_features
        out = {
            "num_data": int(v.num_data), "num_features": nf, "num_total_features": int(v.num_total_features),
            "bins": np.ctypeslib.as_array(v.bins, shape=(int(v.num_data) * nf,)).reshape(int(v.num_data), nf).copy()
            if nf else np.zeros((int(v.num_data), 0), np.uint8),
        }
        for name in ("num_bin", "missing_type", "default_bin", "most_freq_bin", "bin_type", "real_index"):
            out[name] = np.ctypeslib.as_array(getattr(v, name), shape=(nf,)).copy()
        ubo = np.ctypeslib.as_array(v.ub_offsets, shape=(nf + 1,)).copy()
        cao = np.ctypeslib.as_array(v.cat_offsets, shape=(nf + 1,)).copy()
        out["ub_offsets"], out["cat_offsets"] = ubo, cao
        out["upper_bounds"] = (np.ctypeslib.as_array(v.upper_bounds, shape=(int(ubo[-1]),)).copy()
                               if ubo[-1] else np.zeros(0))
        out["bin_to_cat"] = (np.ctypeslib.as_array(v.bin_to_cat, shape=(int(cao[-1]),)).copy()
                             if cao[-1] else np.zeros(0, np.int32))
        return out

    def __del__(self):
        if getattr(self, "_handle", None) is not None and L._lib is not None:
            L._lib.lgbm_b200_dataset_free(self._handle)
            self._handle = None


def tree_from_view(v):
    """A trained tree as a dict of numpy arrays (the reference's Tree fields)."""
    nl = int(v.num_leaves)
    nn = nl - 1

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n > 0 else np.zeros(0, dt)

    t = {"num_leaves": nl}
    for name, n, dt in (("split_feature_inner", nn, np.int32), ("split_feature", nn, np.int32),
                        ("split_gain", nn, np.float32), ("threshold_in_bin", nn, np.uint32),
                        ("threshold", nn, np.float64), ("decision_type", nn, np.int8), ("left_child", nn, np.int32),
                        ("right_child", nn, np.int32), ("leaf_parent", nl, np.int32), ("leaf_value", nl, np.float64),
                        ("leaf_weight", nl, np.float64), ("leaf_count", nl, np.int32), ("leaf_depth", nl, np.int32),
                        ("internal_value", nn, np.float64), ("internal_weight", nn, np.float64),
                        ("internal_count", nn, np.int32)):
        t[name] = arr(getattr(v, name), n, dt)
    nc = int(v.num_cat)
    t["num_cat"] = nc
    t["cat_boundaries"] = arr(v.cat_boundaries, nc + 1, np.int32)
    t["cat_threshold"] = arr(v.cat_threshold, int(t["cat_boundaries"][-1]) if nc else 0, np.uint32)
    t["cat_boundaries_inner"] = arr(v.cat_boundaries_inner, nc + 1, np.int32)
    t["cat_threshold_inner"] = arr(v.cat_threshold_inner, int(t["cat_boundaries_inner"][-1]) if nc else 0,
                                   np.uint32)
    t["split_gain_f64"] = arr(v.split_gain_f64, nn, np.float64) if v.split_gain_f64 else np.zeros(0)
    return t


def _view_from_tree(t, keep):
    """TreeView pointing at the arrays of a tree dict (arrays appended to `keep`)."""
    v = L.TreeView()
    v.num_leaves = t["num_leaves"]
    for name, ct in (("split_feature_inner", C.c_int32), ("split_feature", C.c_int32), ("split_gain", C.c_float),
                     ("threshold_in_bin", C.c_uint32), ("threshold", C.c_double), ("decision_type", C.c_int8),
                     ("left_child", C.c_int32), ("right_child", C.c_int32), ("leaf_parent", C.c_int32),
                     ("leaf_value", C.c_double), ("leaf_weight", C.c_double), ("leaf_count", C.c_int32),
                     ("leaf_depth", C.c_int32), ("internal_value", C.c_double), ("internal_weight", C.c_double),
                     ("internal_count", C.c_int32), ("cat_boundaries", C.c_int32), ("cat_threshold", C.c_uint32),
                     ("cat_boundaries_inner", C.c_int32), ("cat_threshold_inner", C.c_uint32)):
        a = np.ascontiguousarray(t[name])
        if a.size == 0:
            a = np.zeros(1, dtype=a.dtype)
        keep.append(a)
        setattr(v, name, a.ctypes.data_as(C.POINTER(ct)))
    v.num_cat = t["num_cat"]
    return v


def learner_config(p, num_tree_slots=1):
    obj = OBJECTIVES[p["objective"]]
    return L.LearnerConfig(
        int(p["num_leaves"]), int(p["max_depth"]), int(p["min_data_in_leaf"]), float(p["min_sum_hessian_in_leaf"]),
        float(p["lambda_l1"]), float(p["lambda_l2"]), float(p["max_delta_step"]), float(p["path_smooth"]),
        float(p["min_gain_to_split"]), int(p["max_cat_to_onehot"]), int(p["max_cat_threshold"]), float(p["cat_l2"]),
        float(p["cat_smooth"]), int(p["min_data_per_group"]), float(p["monotone_penalty"]),
        HIST[p["hist_precision"]], int(p["num_grad_quant_bins"]), int(bool(p["stochastic_rounding"])),
        int(bool(p["quant_train_renew_leaf"])), int(p["seed"]), int(p["num_threads"]) if p["num_threads"] else 1,
        int(obj == L.OBJ_REGRESSION), int(num_tree_slots), int(p["device"]), int(p["hist_rows_per_block"]), 0,
        int(bool(p["use_cuda_graph"])), int(bool(p["persistent_grow"])))


class Learner:
    """The GPU tree learner over a constructed Dataset (SerialTreeLearner::new)."""

    def __init__(self, train_set, params, num_tree_slots=1):
        self.p = p = resolve_params(params)
        b = train_set.construct(params).binned()
        self.binned = b
        nf = b["num_features"]
        metas = (L.FeatureMeta * max(nf, 1))()
        mono = p.get("monotone_constraints")
        for f in range(nf):
            real = int(b["real_index"][f])
            m = int(mono[real]) if mono is not None and real < len(mono) else 0
            metas[f] = L.FeatureMeta(int(b["num_bin"][f]), int(b["missing_type"][f]), int(b["default_bin"][f]),
                                     int(b["most_freq_bin"][f]), int(b["bin_type"][f]), m, real, 1.0)
        self.cfg = learner_config(p, num_tree_slots)
        h = C.c_void_p()
        bins = np.ascontiguousarray(b["bins"])
        L.check(L.lib().lgbm_b200_learner_create(
            C.byref(self.cfg), _ptr(bins, C.c_uint8), b["num_data"], nf, metas,
            _ptr(b["upper_bounds"], C.c_double) if len(b["upper_bounds"]) else None, _ptr(b["ub_offsets"], C.c_int64),
            _ptr(b["bin_to_cat"], C.c_int32) if len(b["bin_to_cat"]) else None, _ptr(b["cat_offsets"], C.c_int64),
            C.byref(h)))
        self.handle = h
        self.num_tree_slots = num_tree_slots

    def train(self, grad, hess, is_first_tree=False):
        """SerialTreeLearner::train on host gradients; one tree dict per slot."""
        g = np.ascontiguousarray(grad, dtype=np.float32)
        h = np.ascontiguousarray(hess, dtype=np.float32)
        views = (L.TreeView * self.num_tree_slots)()
        L.check(L.lib().lgbm_b200_learner_train(self.handle, g.ctypes.data, h.ctypes.data, int(bool(is_first_tree)),
                                                L.HOST, views))
        return [tree_from_view(views[k]) for k in range(self.num_tree_slots)]

    def set_bagging(self, used):
        if used is None:
            L.check(L.lib().lgbm_b200_learner_set_bagging(self.handle, None, 0, L.HOST))
        else:
            u = np.ascontiguousarray(used, dtype=np.uint32)
            L.check(L.lib().lgbm_b200_learner_set_bagging(self.handle, _ptr(u, C.c_uint32), len(u), L.HOST))

    def set_feature_mask(self, slot, mask):
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        L.check(L.lib().lgbm_b200_learner_set_feature_mask(self.handle, slot,
                                                           _ptr(m, C.c_uint8) if m is not None else None))

    def add_leaf_outputs(self, slot, leaf_values, score):
        lv = np.ascontiguousarray(leaf_values, dtype=np.float64)
        assert score.dtype == np.float64 and score.flags.c_contiguous
        L.check(L.lib().lgbm_b200_learner_add_leaf_outputs(self.handle, slot, _ptr(lv, C.c_double), len(lv),
                                                           score.ctypes.data, L.HOST))

    def partition(self, slot=0, num_leaves=None):
        n = self.binned["num_data"]
        nl = num_leaves or int(self.p["num_leaves"])
        beg = np.zeros(nl, np.int32)
        cnt = np.zeros(nl, np.int32)
        idx = np.zeros(n, np.uint32)
        L.check(L.lib().lgbm_b200_learner_get_partition(self.handle, slot, _ptr(beg, C.c_int32),
                                                        _ptr(cnt, C.c_int32), _ptr(idx, C.c_uint32)))
        return beg, cnt, idx

    def histogram(self, rows=None, slot=0):
        """The learner's histogram kernel over `rows` (diagnostics)."""
        total = int(np.sum(self.binned["num_bin"] - (self.binned["most_freq_bin"] == 0)))
        quant = self.p["hist_precision"] == "quantized"
        out = np.zeros(total if quant else 2 * total, np.int64 if quant else np.float64)
        r = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
        L.check(L.lib().lgbm_b200_learner_histogram(self.handle, slot, _ptr(r, C.c_uint32) if r is not None else None,
                                                    0 if r is None else len(r), out.ctypes.data))
        return out

    def quantized(self, slot=0):
        n = self.binned["num_data"]
        packed = np.zeros(n, np.int64)
        scales = np.zeros(2, np.float64)
        L.check(L.lib().lgbm_b200_learner_quantized(self.handle, slot, _ptr(packed, C.c_int64),
                                                    _ptr(scales, C.c_double)))
        return packed, scales

    def record(self, mark):
        """Record timing mark `mark` (0..15) on the learner's CUDA stream."""
        L.check(L.lib().lgbm_b200_learner_record(self.handle, int(mark)))

    def elapsed(self, a, b):
        """Device milliseconds between two recorded marks."""
        ms = C.c_double()
        L.check(L.lib().lgbm_b200_learner_elapsed(self.handle, int(a), int(b), C.byref(ms)))
        return ms.value

    @property
    def launch_shape(self):
        """The per-step kernels' launch shape: partition_ctas, hist_ctas and
        hist_rows_per_block (dict)."""
        s = L.LaunchShape()
        L.check(L.lib().lgbm_b200_learner_get_launch_shape(self.handle, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in L.LaunchShape._fields_}

    @launch_shape.setter
    def launch_shape(self, shape):
        s = L.LaunchShape(*(int(shape[k]) for k, _ in L.LaunchShape._fields_))
        L.check(L.lib().lgbm_b200_learner_set_launch_shape(self.handle, C.byref(s)))

    def time_shapes(self, shapes, reps=3):
        """Regrow the last train call's trees under each shape (the same
        trees), keep the fastest; returns (index chosen, median ms per tree
        of each shape)."""
        arr = (L.LaunchShape * len(shapes))(*(L.LaunchShape(*(int(sh[k]) for k, _ in L.LaunchShape._fields_))
                                              for sh in shapes))
        ms = (C.c_double * len(shapes))()
        chosen = C.c_int32()
        L.check(L.lib().lgbm_b200_learner_autotune(self.handle, arr, len(shapes), int(reps), C.byref(chosen), ms))
        return int(chosen.value), list(ms)

    def set_timing(self, on):
        L.check(L.lib().lgbm_b200_learner_set_timing(self.handle, int(bool(on))))

    def last_timing(self):
        ms = (C.c_double * 4)()
        rows = C.c_int64()
        launches = C.c_int32()
        L.check(L.lib().lgbm_b200_learner_last_timing(self.handle, ms, C.byref(rows), C.byref(launches)))
        return list(ms), int(rows.value), int(launches.value)

    def set_data_parallel(self, row_offset, global_num_data, allreduce):
        """Grow trees data-parallel: this learner holds rows [row_offset,
        row_offset + its rows) of `global_num_data`, and allreduce(ptr, count,
        dtype, op) reduces a device buffer of this learner's device in place
        over every rank (dtype: L.DT_INT64 / DT_FLOAT64 / DT_INT32; op:
        L.OP_SUM / OP_MAX). See data_parallel.py for torch.distributed ones."""
        def cb(ptr, count, dtype, op, _user):
            try:
                allreduce(ptr, int(count), int(dtype), int(op))
                return 0
            except Exception:  # an exception must not cross the C boundary
                import traceback

                traceback.print_exc()
                return 1

        self._allreduce_cb = L.ALLREDUCE_FN(cb)  # kept alive with the learner
        L.check(L.lib().lgbm_b200_learner_set_data_parallel(self.handle, int(row_offset), int(global_num_data),
                                                            self._allreduce_cb, None))

    def step_times(self):
        """With timing on: (steps x 3) device ms of each split step's
        histogram, scan and partition launches in the last train call."""
        n = C.c_int32()
        L.check(L.lib().lgbm_b200_learner_step_times(self.handle, None, 0, C.byref(n)))
        ms = np.zeros(3 * n.value, np.float32)
        L.check(L.lib().lgbm_b200_learner_step_times(self.handle, _ptr(ms, C.c_float), n.value, C.byref(n)))
        return ms.reshape(-1, 3)

    def last_rows(self):
        """(rows histogrammed, rows partitioned) of the last train call."""
        h, pr = C.c_int64(), C.c_int64()
        L.check(L.lib().lgbm_b200_learner_last_rows(self.handle, C.byref(h), C.byref(pr)))
        return int(h.value), int(pr.value)

    def __del__(self):
        if getattr(self, "handle", None) is not None and L._lib is not None:
            L._lib.lgbm_b200_learner_destroy(self.handle)
            self.handle = None


def objective_config(p):
    obj = OBJECTIVES[p["objective"]]
    return L.ObjectiveConfig(obj, int(p["num_class"]) if obj == L.OBJ_MULTICLASS else 1, float(p["sigmoid"]),
                             int(p["lambdarank_truncation_level"]), int(bool(p["lambdarank_norm"])))


class Objective:
    """An objective bound to its labels once (RowObjective::init): the labels
    stay on the device and gradients() moves only the scores in and g / h out."""

    def __init__(self, params, label, group=None):
        p = resolve_params(params)
        self.label = np.ascontiguousarray(label, dtype=np.float32)
        self.k = int(p["num_class"]) if p["objective"] in ("multiclass", "softmax") else 1
        self.cfg = objective_config(p)
        bnd = None if group is None else np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
        self._bnd = bnd
        h = C.c_void_p()
        L.check(L.lib().lgbm_b200_objective_create(C.byref(self.cfg), self.label.ctypes.data, len(self.label),
                                                   _ptr(bnd, C.c_int32) if bnd is not None else None,
                                                   len(bnd) - 1 if bnd is not None else 0, int(p["device"]),
                                                   C.byref(h)))
        self.handle = h

    def gradients(self, scores, grad=None, hess=None):
        """g, h (float32 [k * n]) of scores (float64 [k * n], class-major)."""
        n = len(self.label) * self.k
        sc = np.ascontiguousarray(scores, dtype=np.float64)
        g = np.empty(n, np.float32) if grad is None else grad
        h = np.empty(n, np.float32) if hess is None else hess
        L.check(L.lib().lgbm_b200_objective_gradients(self.handle, sc.ctypes.data, g.ctypes.data, h.ctypes.data,
                                                      L.HOST))
        return g, h

    def __del__(self):
        if getattr(self, "handle", None):
            L.lib().lgbm_b200_objective_free(self.handle)
            self.handle = None


def metric(name, label, scores, num_class=1, sigmoid=1.0, multi_error_top_k=1, device=0):
    """Metric::eval (metric.rs:520) of host scores on the device: auc,
    binary_logloss, binary_error, l2, rmse, multi_logloss, multi_error
    (unweighted; multiclass scores class-major)."""
    label = np.ascontiguousarray(label, dtype=np.float32)
    scores = np.ascontiguousarray(scores, dtype=np.float64)
    cfg = L.MetricConfig(L.METRICS[name], int(num_class), float(sigmoid), int(multi_error_top_k))
    out = C.c_double()
    L.check(L.lib().lgbm_b200_metric_eval(C.byref(cfg), _ptr(label, C.c_float), _ptr(scores, C.c_double), len(label),
                                          L.HOST, int(device), C.byref(out)))
    return out.value


def ndcg(label, scores, group, eval_at, device=0):
    """NDCG@k for each k of eval_at on the device (metric.rs:546-598);
    `group` holds the query sizes."""
    label = np.ascontiguousarray(label, dtype=np.float32)
    scores = np.ascontiguousarray(scores, dtype=np.float64)
    bnd = np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
    ks = np.ascontiguousarray(eval_at, dtype=np.int32)
    out = np.zeros(len(ks), np.float64)
    L.check(L.lib().lgbm_b200_metric_ndcg(_ptr(label, C.c_float), _ptr(scores, C.c_double), _ptr(bnd, C.c_int32),
                                          len(bnd) - 1, _ptr(ks, C.c_int32), len(ks), L.HOST, int(device),
                                          _ptr(out, C.c_double)))
    return out


def gradients(params, label, scores, group=None):
    """RowObjective::gradients on the GPU from host arrays."""
    p = resolve_params(params)
    oc = objective_config(p)
    label = np.ascontiguousarray(label, dtype=np.float32)
    scores = np.ascontiguousarray(scores, dtype=np.float64)
    g = np.empty(scores.shape, np.float32)
    h = np.empty(scores.shape, np.float32)
    bnd = None
    nq = 0
    if group is not None:
        bnd = np.concatenate([[0], np.cumsum(group)]).astype(np.int32)
        nq = len(group)
    L.check(L.lib().lgbm_b200_gradients(C.byref(oc), label.ctypes.data, scores.ctypes.data, len(label),
                                        _ptr(bnd, C.c_int32) if bnd is not None else None, nq, g.ctypes.data,
                                        h.ctypes.data, L.HOST, int(p["device"])))
    return g, h


class Booster:
    """A model trained on the device (python/lightgbm_rust/basic.py:1364)."""

    def __init__(self, params=None, train_set=None, valid_set=None):
        self.params = resolve_params(params)
        p = self.params
        self.num_class = int(p["num_class"]) if OBJECTIVES[p["objective"]] == L.OBJ_MULTICLASS else 1
        self.trees = []
        self.shrinkages = []  # Tree::shrinkage of each tree (tree.rs:303-339)
        self._forest = None
        self.learner = None
        self._b = None
        self._train_set = train_set
        if train_set is not None:
            self.learner = Learner(train_set, params, num_tree_slots=self.num_class)
            valid_bins = None
            nv = 0
            if valid_set is not None:
                vb = valid_set.construct(params).binned()
                valid_bins = np.ascontiguousarray(vb["bins"])
                nv = vb["num_data"]
                self._valid_bins = valid_bins
            bc = L.BoostConfig(objective_config(p), float(p["learning_rate"]), int(bool(p["boost_from_average"])),
                               float(p["bagging_fraction"]), int(p["bagging_freq"]), int(p["bagging_seed"]),
                               float(p["feature_fraction"]), int(p["feature_fraction_seed"]))
            label = np.ascontiguousarray(train_set.label, dtype=np.float32)
            bnd = None
            if train_set.group is not None:  # query boundaries (dataset.rs set_group)
                bnd = np.concatenate([[0], np.cumsum(train_set.group)]).astype(np.int32)
                self._bnd = bnd
            h = C.c_void_p()
            L.check(L.lib().lgbm_b200_booster_create(
                self.learner.handle, C.byref(bc), _ptr(label, C.c_float), _ptr(bnd, C.c_int32) if bnd is not None
                else None, 0 if bnd is None else len(bnd) - 1,
                _ptr(valid_bins, C.c_uint8) if valid_bins is not None else None, nv, C.byref(h)))
            self._b = h
            self.num_train = train_set.data.shape[0]
            self.num_valid = nv

    def update(self):
        """One boosting iteration (Booster.update); returns True when training stopped."""
        stop = C.c_int32()
        views = (L.TreeView * self.num_class)()
        L.check(L.lib().lgbm_b200_booster_train_iter(self._b, C.byref(stop), views))
        if stop.value:
            return True
        first = not self.trees
        if first:
            init = np.zeros(self.num_class, np.float64)
            L.check(L.lib().lgbm_b200_booster_init_scores(self._b, _ptr(init, C.c_double)))
        for k in range(self.num_class):
            t = tree_from_view(views[k])
            self.trees.append(t)
            # shrink() multiplies the shrinkage by the learning rate; add_bias
            # (the first iteration's boost_from_average score) and a constant
            # tree set it back to 1
            if t["num_leaves"] <= 1 or (first and abs(init[k]) > model_text.K_EPSILON):
                self.shrinkages.append(1.0)
            else:
                self.shrinkages.append(float(self.params["learning_rate"]))
        self._forest = None
        return False

    def model_to_string(self):
        """Gbdt::save_model_to_string (io.rs:13-85): the model text from the
        header through the feature importances (model_text.py)."""
        ds = self._train_set
        if ds is None:
            raise L.LightGBMError(L.ERR_INVALID_PARAMETER, "model_to_string needs the training Dataset")
        ds.construct(self.params)
        infos = C.c_char_p()
        L.check(L.lib().lgbm_b200_dataset_feature_infos(ds._handle, C.byref(infos)))
        mono = self.params.get("monotone_constraints")
        return model_text.model_to_string(self.params, self.trees, self.shrinkages, self.num_class,
                                          ds.data.shape[1], infos.value.decode().split(" "), mono)

    def save_model(self, filename):
        with open(filename, "w") as f:
            f.write(self.model_to_string())
        return self

    def scores(self, valid=False):
        n = self.num_valid if valid else self.num_train
        out = np.zeros(self.num_class * n, np.float64)
        L.check(L.lib().lgbm_b200_booster_scores(self._b, 1 if valid else 0, out.ctypes.data, L.HOST))
        return out.reshape(self.num_class, n)

    def num_trees(self):
        return len(self.trees)

    def _forest_handle(self):
        if self._forest is None:
            keep = []
            views = (L.TreeView * max(1, len(self.trees)))()
            for i, t in enumerate(self.trees):
                views[i] = _view_from_tree(t, keep)
            h = C.c_void_p()
            L.check(L.lib().lgbm_b200_forest_create(views, len(self.trees), self.num_class, int(self.params["device"]),
                                                    C.byref(h)))
            self._forest = h
        return self._forest

    def predict(self, data, raw_score=False):
        """Gbdt::predict_matrix_early_stop (raw, then the objective's transform)."""
        X = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
        out = np.zeros(X.shape[0] * self.num_class, np.float64)
        L.check(L.lib().lgbm_b200_predict(self._forest_handle(), X.ctypes.data, X.shape[0], X.shape[1],
                                          out.ctypes.data, L.HOST))
        raw = out.reshape(X.shape[0], self.num_class)
        if raw_score:
            return raw[:, 0] if self.num_class == 1 else raw
        obj = OBJECTIVES[self.params["objective"]]
        if obj == L.OBJ_BINARY:  # binary.rs:164-166
            return 1.0 / (1.0 + np.exp(-float(self.params["sigmoid"]) * raw[:, 0]))
        if obj == L.OBJ_MULTICLASS:  # multiclass.rs:165-167 softmax
            e = np.exp(raw - raw.max(axis=1, keepdims=True))
            return e / e.sum(axis=1, keepdims=True)
        return raw[:, 0]

    def __del__(self):
        if L._lib is None:
            return
        if getattr(self, "_forest", None) is not None:
            L._lib.lgbm_b200_forest_destroy(self._forest)
            self._forest = None
        if getattr(self, "_b", None) is not None:
            L._lib.lgbm_b200_booster_destroy(self._b)
            self._b = None


def train(params, train_set, num_boost_round=100, valid_sets=None):
    """engine.py:50 train: boosting on the device, one tree set per iteration."""
    p = dict(params or {})
    nbr = p.pop("num_boost_round", None) or num_boost_round
    valid = valid_sets[0] if valid_sets else None
    bst = Booster(p, train_set, valid)
    for _ in range(int(nbr)):
        if bst.update():
            break
    return bst
