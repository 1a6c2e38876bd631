"""Builds liblgbm_b200.so and liblgbm_b200.a (CUDA kernels for sm_100a +
host C++) in-tree.

Usage: python lightgbm-rust_b200/build.py [--clean]
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "lgbm_b200", "liblgbm_b200.so")
STATIC = os.path.join(HERE, "lgbm_b200", "liblgbm_b200.a")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: every a*b+c stays a rounded multiply and a rounded add, as on
# the reference's CPU path, so split gains match bit for bit.
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-fopenmp,-O2",
           "-I" + os.path.join(HERE, "..", "include")]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-I/usr/local/cuda/include",
            "-I" + os.path.join(HERE, "..", "include")]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose=False, extra_nvcc=()):
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "lgbm_b200.h"))
    jobs = []
    objs = []
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            jobs.append([NVCC] + ARCH + NVFLAGS + list(extra_nvcc) + ["-c", src, "-o", obj])
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            jobs.append(["g++"] + CXXFLAGS + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("compile failed: " + cmd[-3])
    if jobs or not os.path.exists(OUT):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lgomp", "-Xcompiler", "-fopenmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if jobs or not os.path.exists(STATIC):
        # the same objects as a static archive, for a Rust build.rs that links
        # `static=lgbm_b200` with `static=cudart_static` (every .cu file is
        # compiled whole, so no device-link step is needed)
        if os.path.exists(STATIC):
            os.remove(STATIC)
        r = subprocess.run(["ar", "rcs", STATIC] + objs, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("archive failed")
    return OUT


if __name__ == "__main__":
    if "--clean" in sys.argv:
        shutil.rmtree(BUILD, ignore_errors=True)
    print(build(verbose="-v" in sys.argv))
