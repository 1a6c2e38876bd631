"""ctypes bindings of liblgbm_b200.so (include/lgbm_b200.h).

The shared library is built in-tree by ``lightgbm-rust_b200/build.py``; the
package refuses to work without it (there is no CPU fallback).
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# LGBM_B200_LIB names another build of the library (for example one compiled
# with a different partition tile size)
LIB_PATH = os.environ.get("LGBM_B200_LIB") or os.path.join(_HERE, "liblgbm_b200.so")

OK = 0
ERR_INVALID_PARAMETER = 1
ERR_INVALID_DATA = 2
ERR_MODEL_FORMAT = 3
ERR_UNSUPPORTED = 4
ERR_INTERNAL = 5
ERR_CUDA = 6
ERR_TIMEOUT = 7
HOST = 0
DEVICE = 1
HIST_F64 = 0
HIST_F32C = 1
HIST_QUANT = 2
OBJ_BINARY = 0
OBJ_REGRESSION = 1
OBJ_MULTICLASS = 2
OBJ_LAMBDARANK = 3

i32, i64, f64, u8p = C.c_int32, C.c_int64, C.c_double, C.POINTER(C.c_uint8)
P = C.POINTER


class BinParams(C.Structure):
    _fields_ = [("max_bin", i32), ("min_data_in_bin", i32), ("min_data_in_leaf", i32),
                ("bin_construct_sample_cnt", i32), ("data_random_seed", i32), ("use_missing", i32),
                ("zero_as_missing", i32), ("feature_pre_filter", i32), ("categorical", P(i32)),
                ("num_categorical", i32)]


class MetricConfig(C.Structure):
    _fields_ = [("metric", i32), ("num_class", i32), ("sigmoid", f64), ("multi_error_top_k", i32)]


METRICS = {"auc": 0, "binary_logloss": 1, "binary_error": 2, "l2": 3, "rmse": 4, "multi_logloss": 5,
           "multi_error": 6}


class DatasetView(C.Structure):
    _fields_ = [("num_data", i64), ("num_features", i32), ("num_total_features", i32), ("bins", u8p),
                ("num_bin", P(i32)), ("missing_type", P(i32)), ("default_bin", P(i32)),
                ("most_freq_bin", P(i32)), ("bin_type", P(i32)), ("real_index", P(i32)),
                ("upper_bounds", P(f64)), ("ub_offsets", P(i64)), ("bin_to_cat", P(i32)),
                ("cat_offsets", P(i64))]


class LearnerConfig(C.Structure):
    _fields_ = [("num_leaves", i32), ("max_depth", i32), ("min_data_in_leaf", i32),
                ("min_sum_hessian_in_leaf", f64), ("lambda_l1", f64), ("lambda_l2", f64),
                ("max_delta_step", f64), ("path_smooth", f64), ("min_gain_to_split", f64),
                ("max_cat_to_onehot", i32), ("max_cat_threshold", i32), ("cat_l2", f64), ("cat_smooth", f64),
                ("min_data_per_group", i32), ("monotone_penalty", f64), ("hist_precision", i32),
                ("num_grad_quant_bins", i32), ("stochastic_rounding", i32), ("quant_train_renew_leaf", i32),
                ("seed", i32), ("quant_num_threads", i32), ("is_constant_hessian", i32),
                ("num_tree_slots", i32), ("device", i32), ("hist_rows_per_block", i32),
                ("hist_block_threads", i32), ("use_cuda_graph", i32), ("persistent_grow", i32)]


class FeatureMeta(C.Structure):
    _fields_ = [("num_bin", i32), ("missing_type", i32), ("default_bin", i32), ("most_freq_bin", i32),
                ("bin_type", i32), ("monotone_type", i32), ("real_index", i32), ("penalty", f64)]


class TreeView(C.Structure):
    _fields_ = [("num_leaves", i32), ("split_feature_inner", P(i32)), ("split_feature", P(i32)),
                ("split_gain", P(C.c_float)), ("threshold_in_bin", P(C.c_uint32)), ("threshold", P(f64)),
                ("decision_type", P(C.c_int8)), ("left_child", P(i32)), ("right_child", P(i32)),
                ("leaf_parent", P(i32)), ("leaf_value", P(f64)), ("leaf_weight", P(f64)), ("leaf_count", P(i32)),
                ("leaf_depth", P(i32)), ("internal_value", P(f64)), ("internal_weight", P(f64)),
                ("internal_count", P(i32)), ("num_cat", i32), ("cat_boundaries", P(i32)),
                ("cat_threshold", P(C.c_uint32)), ("cat_boundaries_inner", P(i32)),
                ("cat_threshold_inner", P(C.c_uint32)), ("split_gain_f64", P(f64))]


class ObjectiveConfig(C.Structure):
    _fields_ = [("objective", i32), ("num_class", i32), ("sigmoid", f64), ("lambdarank_truncation_level", i32),
                ("lambdarank_norm", i32)]


class BoostConfig(C.Structure):
    _fields_ = [("objective", ObjectiveConfig), ("learning_rate", f64), ("boost_from_average", i32),
                ("bagging_fraction", f64), ("bagging_freq", i32), ("bagging_seed", i32),
                ("feature_fraction", f64), ("feature_fraction_seed", i32)]


class LaunchShape(C.Structure):
    _fields_ = [("partition_ctas", i32), ("hist_ctas", i32), ("hist_rows_per_block", i32)]


# the data-parallel reduction callback: (device buffer, count, dtype, op, user) -> 0 on success
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, i64, i32, i32, C.c_void_p)
DT_INT64, DT_FLOAT64, DT_INT32 = 0, 1, 2
OP_SUM, OP_MAX = 0, 1

# name -> (restype, argtypes)
SIGNATURES = {
    "lgbm_b200_last_error": (C.c_char_p, []),
    "lgbm_b200_version": (C.c_char_p, []),
    "lgbm_b200_dataset_create": (C.c_int, [P(C.c_float), i64, i32, P(BinParams), P(C.c_void_p)]),
    "lgbm_b200_dataset_create_valid": (C.c_int, [P(C.c_float), i64, i32, C.c_void_p, P(C.c_void_p)]),
    "lgbm_b200_metric_eval": (C.c_int, [P(MetricConfig), P(C.c_float), P(f64), i64, i32, i32, P(f64)]),
    "lgbm_b200_metric_ndcg": (C.c_int, [P(C.c_float), P(f64), P(i32), i32, P(i32), i32, i32, i32, P(f64)]),
    "lgbm_b200_dataset_create_device": (C.c_int, [P(C.c_float), i64, i32, P(BinParams), i32, P(C.c_void_p)]),
    "lgbm_b200_dataset_create_valid_device": (C.c_int, [P(C.c_float), i64, i32, C.c_void_p, i32, P(C.c_void_p)]),
    "lgbm_b200_dataset_view": (C.c_int, [C.c_void_p, P(DatasetView)]),
    "lgbm_b200_dataset_feature_infos": (C.c_int, [C.c_void_p, P(C.c_char_p)]),
    "lgbm_b200_dataset_free": (None, [C.c_void_p]),
    "lgbm_b200_learner_create": (C.c_int, [P(LearnerConfig), u8p, i64, i32, P(FeatureMeta), P(f64), P(i64),
                                           P(i32), P(i64), P(C.c_void_p)]),
    "lgbm_b200_learner_destroy": (None, [C.c_void_p]),
    "lgbm_b200_learner_set_bagging": (C.c_int, [C.c_void_p, P(C.c_uint32), i64, i32]),
    "lgbm_b200_learner_set_feature_mask": (C.c_int, [C.c_void_p, i32, u8p]),
    "lgbm_b200_learner_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, i32, i32, P(TreeView)]),
    "lgbm_b200_learner_add_leaf_outputs": (C.c_int, [C.c_void_p, i32, P(f64), i32, C.c_void_p, i32]),
    "lgbm_b200_learner_get_partition": (C.c_int, [C.c_void_p, i32, P(i32), P(i32), P(C.c_uint32)]),
    "lgbm_b200_learner_get_launch_shape": (C.c_int, [C.c_void_p, P(LaunchShape)]),
    "lgbm_b200_learner_set_launch_shape": (C.c_int, [C.c_void_p, P(LaunchShape)]),
    "lgbm_b200_learner_autotune": (C.c_int, [C.c_void_p, P(LaunchShape), i32, i32, P(i32), P(f64)]),
    "lgbm_b200_learner_set_timing": (C.c_int, [C.c_void_p, i32]),
    "lgbm_b200_learner_last_timing": (C.c_int, [C.c_void_p, P(f64), P(i64), P(i32)]),
    "lgbm_b200_learner_last_rows": (C.c_int, [C.c_void_p, P(i64), P(i64)]),
    "lgbm_b200_learner_step_times": (C.c_int, [C.c_void_p, P(C.c_float), i32, P(i32)]),
    "lgbm_b200_learner_set_data_parallel": (C.c_int, [C.c_void_p, i64, i64, ALLREDUCE_FN, C.c_void_p]),
    "lgbm_b200_learner_record": (C.c_int, [C.c_void_p, i32]),
    "lgbm_b200_learner_elapsed": (C.c_int, [C.c_void_p, i32, i32, P(f64)]),
    "lgbm_b200_learner_histogram": (C.c_int, [C.c_void_p, i32, P(C.c_uint32), i64, C.c_void_p]),
    "lgbm_b200_learner_quantized": (C.c_int, [C.c_void_p, i32, P(i64), P(f64)]),
    "lgbm_b200_objective_create": (C.c_int, [P(ObjectiveConfig), C.c_void_p, i64, P(i32), i32, i32,
                                             P(C.c_void_p)]),
    "lgbm_b200_objective_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, i32]),
    "lgbm_b200_objective_free": (None, [C.c_void_p]),
    "lgbm_b200_gradients": (C.c_int, [P(ObjectiveConfig), C.c_void_p, C.c_void_p, i64, P(i32), i32, C.c_void_p,
                                      C.c_void_p, i32, i32]),
    "lgbm_b200_booster_create": (C.c_int, [C.c_void_p, P(BoostConfig), P(C.c_float), P(i32), i32, u8p, i64,
                                           P(C.c_void_p)]),
    "lgbm_b200_booster_destroy": (None, [C.c_void_p]),
    "lgbm_b200_booster_train_iter": (C.c_int, [C.c_void_p, P(i32), P(TreeView)]),
    "lgbm_b200_booster_scores": (C.c_int, [C.c_void_p, i32, C.c_void_p, i32]),
    "lgbm_b200_booster_init_scores": (C.c_int, [C.c_void_p, P(f64)]),
    "lgbm_b200_forest_create": (C.c_int, [P(TreeView), i32, i32, i32, P(C.c_void_p)]),
    "lgbm_b200_forest_destroy": (None, [C.c_void_p]),
    "lgbm_b200_predict": (C.c_int, [C.c_void_p, C.c_void_p, i64, i32, C.c_void_p, i32]),
    "lgbm_b200_predict_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, i64, i32, C.c_void_p]),
}

_lib = None


class LightGBMError(Exception):
    """Error raised by the library (the reference's LgbmError kinds)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"liblgbm_b200.so not found at {LIB_PATH}: run lightgbm-rust_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != OK:
        msg = lib().lgbm_b200_last_error()
        raise LightGBMError(rc, msg.decode() if msg else f"error {rc}")
