"""Element-tile autotuner: picks the cells per CTA of the stage kernel.

The fused stage kernel stages ``cells_per_cta`` cells in shared memory; the
best tile depends on N, the arithmetic form and the mesh size (occupancy
against barrier stalls and the tail of the grid).  ``tune`` times each
candidate on the caller's own case for a few RK3 steps and keeps the
fastest; results are cached per (GPU, N, form, size class) in
``sddc_b200/lib/autotune.json``.
"""
from __future__ import annotations

import json
import math
import os
import time

from . import _native
from .solver import Solver

CANDIDATES = (4, 6, 8, 16)
CACHE = os.path.join(_native.LIB_DIR, "autotune.json")


def _key(N, precision, ncell, device_name):
    return f"{device_name}|N{N}|{precision}|2^{int(math.log2(max(ncell, 1)))}"


def _device_name():
    # the cache lives beside the build of one machine; a different GPU model
    # is told apart by the SDDC_DEVICE environment variable when needed
    return os.environ.get("SDDC_DEVICE", "gpu")


def load_cache() -> dict:
    try:
        return json.load(open(CACHE))
    except Exception:
        return {}


def tune(tables, physics, Q0, dt, precision="mixed", steps=3, candidates=CANDIDATES, use_cache=True):
    """Returns (best cells_per_cta, {cpb: seconds per step})."""
    key = _key(tables.N, precision, tables.ncell, _device_name())
    cache = load_cache()
    if use_cache and key in cache:
        return int(cache[key]["best"]), cache[key]["times"]
    times = {}
    for cpb in candidates:
        s = Solver(tables, physics, precision=precision, cells_per_cta=cpb)
        s.set_state(Q0)
        s.rk_s5p3(dt, 2)  # first step eager, second captures the graph
        t0 = time.perf_counter()
        s.rk_s5p3(dt, steps)
        times[cpb] = (time.perf_counter() - t0) / steps
        s.close()
    best = min(times, key=times.get)
    cache[key] = {"best": best, "times": {str(k): v for k, v in times.items()}}
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        json.dump(cache, open(CACHE, "w"), indent=1)
    except OSError:
        pass
    return best, times
