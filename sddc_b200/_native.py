"""Locating and loading the package's native libraries.

Both libraries are built in-tree (``sddc_b200/lib/``) by ``sddc_b200.build``.
A missing library is an error, never a silent fallback: the solver has no CPU
path.
"""
from __future__ import annotations

import ctypes
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
HOST_LIB = os.path.join(LIB_DIR, "libsddc_host.so")
GPU_LIB = os.path.join(LIB_DIR, "libsddc_b200.so")

_cache: dict[str, ctypes.CDLL] = {}


class NativeLibraryMissing(RuntimeError):
    pass


def load(path: str) -> ctypes.CDLL:
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{os.path.basename(path)} is not built ({path}); run `python -m sddc_b200.build`")
    lib = ctypes.CDLL(path)
    _cache[path] = lib
    return lib


def ptr(a, ctype=ctypes.c_double):
    """ctypes pointer to the data of a numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))
