"""The C ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(lgbm_b200_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(lgb):
    names = _declared()
    assert len(names) > 20
    lib = C.CDLL(lgb._lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_gpu(lgb):
    L = lgb.lib()
    assert b"sm_100a" in L.lgbm_b200_version()
    # a host-only error path: bad arguments are rejected before any CUDA call
    rc = L.lgbm_b200_dataset_create(None, 0, 0, None, None)
    assert rc == lgb._lib.ERR_INVALID_PARAMETER
    assert L.lgbm_b200_last_error()


def test_bindings_cover_the_header(lgb):
    names = _declared()
    bound = set(lgb._lib.SIGNATURES)
    assert names <= bound, sorted(names - bound)
