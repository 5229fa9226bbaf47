"""Build the native libraries of taco_b200 in-tree.

* libtaco_b200.so  -- the C-ABI library (include/taco_b200.h): sm_100a CUDA kernels and
                      the host orchestration, compiled by nvcc.
* _taco_native*.so -- the pybind11 module wrapping the same C-ABI.

Usage:  python -m taco_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libtaco_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("TACO_NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = os.environ.get("TACO_HOST_CXX", "g++")

LIB_SOURCES = ["engine.cu", "guard.cu", "noalloc.cu", "tcl2.cu", "mikx_gw.cu", "bcf.cu", "adjoint.cu", "capi.cpp", "gw_coef.cpp"]


def _native_ext() -> str:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.join(PKG, "_taco_native" + suffix)


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    return (glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h"))
            + [os.path.abspath(__file__)])


def build_lib(force: bool = False, verbose: bool = False) -> str:
    """Compile the sources to objects in parallel (one nvcc per source), then link."""
    if not force and not _stale(LIB, _deps()):
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(ROOT, "_build", "lib")
    os.makedirs(objdir, exist_ok=True)
    common = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
              "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr"]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in LIB_SOURCES]

    def compile_one(k):
        subprocess.run([*common, "-c", os.path.join(CSRC, LIB_SOURCES[k]), "-o", objs[k]], check=True)

    with ThreadPoolExecutor(max_workers=min(len(LIB_SOURCES), os.cpu_count() or 1)) as pool:
        list(pool.map(compile_one, range(len(LIB_SOURCES))))
    subprocess.run([NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-o", LIB, *objs, "-lcudart"], check=True)
    return LIB


def build_native(force: bool = False) -> str:
    import pybind11

    out = _native_ext()
    src = os.path.join(CSRC, "taco_native.cpp")
    if not force and not _stale(out, [src, LIB, os.path.join(INCLUDE, "taco_b200.h")]):
        return out
    py_inc = sysconfig.get_paths()["include"]
    cmd = [HOST_CXX, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", INCLUDE, "-I", pybind11.get_include(),
           "-I", py_inc, src, "-o", out, "-L", PKG, "-ltaco_b200", "-Wl,-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    return out


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force, verbose)
    build_native(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
