"""lgbm_b200: a B200 (sm_100a) tree-learning path for lightgbm-rust.

The CUDA kernels and the C ABI live in liblgbm_b200.so (include/lgbm_b200.h);
this package is the host-side harness that mirrors lightgbm-rust's Python
API for the path: Dataset, Booster, train.
"""
from ._lib import LightGBMError, lib  # noqa: F401
from .basic import Booster, Dataset, Learner, Objective, gradients, metric, ndcg, resolve_params, train  # noqa: F401

__all__ = ["Booster", "Dataset", "Learner", "LightGBMError", "Objective", "gradients", "lib", "metric", "ndcg", "resolve_params", "train"]
