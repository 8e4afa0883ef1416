"""In-tree build of the sm_100a CUDA library ``_lib/libtdscha_b200.so`` with nvcc.

Every .cu under ``python-sscha_b200/csrc`` is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one shared library
(static CUDA runtime, cuBLAS for the FP64 library GEMMs).  Rebuilds only when a source or header
is newer than the library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                      # python-sscha_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIB_DIR = os.path.join(PKG_DIR, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libtdscha_b200.so")
DRIVER_SRC = os.path.join(ROOT, "driver", "tdscha_lanczos_b200.cpp")
DRIVER_PATH = os.path.join(LIB_DIR, "tdscha_lanczos_b200")
OBJ_DIR = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib_dir():
    nv = _nvcc()
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nv))), "lib64")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    """Compile and link the library; returns its path."""
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    nvcc = _nvcc()
    objs = []
    for src in sources():
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc] + NVCC_FLAGS + ["-I", CSRC, "-I", INCLUDE, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB_PATH, objs):
        libdir = _cuda_lib_dir()
        cmd = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB_PATH] + objs + [
            "-L", libdir, "-lcublas", "-Xlinker", f"-rpath={libdir}"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    build_driver(verbose=verbose, force=force)
    return LIB_PATH


def build_driver(verbose=False, force=False):
    """The stand-alone Lanczos program (driver/tdscha_lanczos_b200.cpp), linked against the library."""
    deps = [DRIVER_SRC, LIB_PATH] + glob.glob(os.path.join(INCLUDE, "*.h"))
    if force or _stale(DRIVER_PATH, deps):
        cmd = [_nvcc(), "-std=c++17", "-O2"] + ARCH + ["-I", INCLUDE, DRIVER_SRC, "-o", DRIVER_PATH, "-L", LIB_DIR, "-ltdscha_b200",
               "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return DRIVER_PATH


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
