"""Builds the package's native libraries in-tree (``sddc_b200/lib``).

* ``libsddc_host.so``: host set-up (g++, no CUDA);
* ``libsddc_b200.so``: the drop-in, CUDA for sm_100a.  The exact FP64 form
  is compiled in its own translation unit with ``-fmad=false`` so that no
  multiply-add is contracted; the other forms keep contraction.

Usage: ``python -m sddc_b200.build [--force]``.  Objects are rebuilt when a
source or header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "lib", "obj")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
               f"-I{INCLUDE}", f"-I{CSRC}"]
CUDA_UNITS = {
    "stage_exact.cu": ["-fmad=false"],
    "stage_fp64.cu": [],
    # single-precision divide and square root of the mixed form's flux work
    # to the hardware approximations (within 2 ulp); FP64 is unaffected
    "stage_mixed.cu": ["-prec-div=false", "-prec-sqrt=false"],
    "context.cu": [],
    "noalloc.cu": [],
    "adjoint.cu": [],
    "adjoint_exact.cu": ["-fmad=false"],
    "output.cu": ["-fmad=false"],
}


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _newest_dep() -> float:
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _stale(target: str, dep_time: float) -> bool:
    return not os.path.exists(target) or os.path.getmtime(target) < dep_time


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_host(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libsddc_host.so")
    if force or _stale(out, _newest_dep()):
        _run([_cxx(), "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-Wall",
              f"-I{INCLUDE}", "-o", out, os.path.join(CSRC, "host_setup.cpp")])
    return out


def build_gpu(force: bool = False, jobs: int = 4) -> str:
    os.makedirs(OBJ, exist_ok=True)
    out = os.path.join(LIB, "libsddc_b200.so")
    dep = _newest_dep()
    nvcc = _nvcc()

    def compile_unit(name):
        obj = os.path.join(OBJ, name.replace(".cu", ".o"))
        if force or _stale(obj, dep):
            _run([nvcc, *ARCH, *NVCC_COMMON, *CUDA_UNITS[name], "-c", os.path.join(CSRC, name), "-o", obj])
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_unit, CUDA_UNITS))
    if force or _stale(out, max(os.path.getmtime(o) for o in objs)):
        _run([nvcc, *ARCH, "-shared", "-o", out, *objs, "-lcudart"])
    return out


def build_oracle() -> str:
    """The CPU oracle is test infrastructure; built here so tests find it."""
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return os.path.join(ROOT, "oracle", "libsddc_oracle.so")


def build_all(force: bool = False) -> list[str]:
    return [build_host(force), build_gpu(force), build_oracle()]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
