"""Test configuration: paths, the `gpu` marker, shared fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's known
answers, the host-side code and the C ABI's exports; GPU tests (-m gpu)
compare the CUDA path with the oracle through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "lightgbm-rust_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """liblgbm_b200.so and the oracle, built in-tree (cached by mtime)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("lgbm_b200_build", os.path.join(ROOT, "lightgbm-rust_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)

    if not os.environ.get("LGBM_B200_SKIP_BUILD"):
        b.build()
    from oracle import oracle

    oracle.build()
    return True


@pytest.fixture(scope="session")
def lgb(built):
    import lgbm_b200

    return lgbm_b200


@pytest.fixture(scope="session")
def orc(built):
    from oracle import oracle

    return oracle


def binned_dataset(lgb, X, y=None, params=None, reference=None, categorical=None):
    ds = lgb.Dataset(X, label=y, params=params, reference=reference, categorical_feature=categorical)
    ds.construct(params)
    return ds
