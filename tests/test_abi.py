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


def test_static_archive_links_a_c_program(lgb, tmp_path):
    """liblgbm_b200.a (what a Rust build.rs links with static=lgbm_b200 and
    static=cudart_static) holds every declared entry point, and a C program
    linked against it alone runs a host-only call."""
    import subprocess

    archive = os.path.join(os.path.dirname(lgb._lib.LIB_PATH), "liblgbm_b200.a")
    assert os.path.exists(archive)
    out = subprocess.run(["nm", "-g", "--defined-only", archive], capture_output=True, text=True, check=True).stdout
    defined = set(re.findall(r"\bT (lgbm_b200_[a-z0-9_]+)\b", out))
    missing = sorted(_declared() - defined)
    assert not missing, missing
    src = tmp_path / "main.c"
    src.write_text('#include <stdio.h>\n#include "lgbm_b200.h"\n'
                   'int main(void) { puts(lgbm_b200_version());\n'
                   '  return lgbm_b200_dataset_create(0, 0, 0, 0, 0) == LGBM_B200_ERR_INVALID_PARAMETER ? 0 : 1; }\n')
    exe = tmp_path / "main"
    subprocess.run(["gcc", "-c", str(src), "-I", os.path.join(ROOT, "include"), "-o", str(tmp_path / "main.o")],
                   check=True)
    subprocess.run(["g++", str(tmp_path / "main.o"), archive, "-L/usr/local/cuda/lib64", "-lcudart_static",
                    "-lgomp", "-lpthread", "-ldl", "-lrt", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "sm_100a" in r.stdout
