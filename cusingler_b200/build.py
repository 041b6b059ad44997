"""In-tree build of the native library and the drop-in Python module.

* ``cusingler_b200/_lib/libsgr.so``: the C ABI of ``include/sgr.h`` (CUDA for sm_100a + host C++).
* ``cusingler/cusingler<ext>``: the pybind11 module with the reference's ``run(...)`` signature,
  importable as ``from cusingler import cusingler`` like the reference's wheel.

nvcc cross-compiles without a GPU.  Objects are rebuilt only when a source or header is newer.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(LIBDIR, "libsgr.so")
MODDIR = os.path.join(ROOT, "cusingler")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", *ARCH]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        if os.path.basename(src) == "pymodule.cpp":
            continue
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            if src.endswith(".cu"):
                _run([NVCC, *NVFLAGS, "-c", src, "-o", obj], verbose)
            else:
                _run([NVCC, "-x", "cu", *NVFLAGS, "-c", src, "-o", obj], verbose)
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"], verbose)
    return LIB


def build_module(verbose: bool = False) -> str:
    import pybind11

    os.makedirs(MODDIR, exist_ok=True)
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(MODDIR, "cusingler" + ext)
    src = os.path.join(CSRC, "pymodule.cpp")
    if _stale(out, [src, LIB, os.path.join(ROOT, "include", "sgr.h")]):
        _run(["g++", *CXXFLAGS, "-shared", src, "-o", out,
              "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
              "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lsgr",
              "-Wl,-rpath,$ORIGIN/../cusingler_b200/_lib"], verbose)
    return out


def build(verbose: bool = False) -> None:
    build_lib(verbose)
    build_module(verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
