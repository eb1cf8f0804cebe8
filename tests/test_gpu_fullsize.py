"""Parity and size-independent properties at the benchmark's full size
(cylinder 256 x 512, p = 4: 3.3M solution points x 9 variables)."""
import math
import os

import numpy as np
import pytest

import sddc_oracle as O
from helpers import rel_l2
from sddc_b200 import cases, host
from sddc_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    c = cases.cylinder_case(256, 512, 5, ms=0.5, ma=2.0, seed=0, noise=1e-6)
    t = host.build_tables(c.mesh, c.N)
    Q0 = c.initial_state(t)
    dt = cases.cfl_dt(c.mesh, Q0, c.N)
    return c, t, Q0, dt


def test_fullsize_exact_equals_oracle(big):
    """Two RK3 steps of the full case: the exact form is bit-equal to the
    CPU oracle."""
    c, t, Q0, dt = big
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(t, c.physics)
    o.set_state(Q0)
    o.rk_s5p3(dt, 2)
    s = Solver(t, c.physics, precision="fp64_exact")
    s.set_state(Q0)
    s.rk_s5p3(dt, 2)
    assert np.array_equal(s.state()["Q"], o.state()["Q"])
    mo, mg = o.maxima(), s.maxima()
    assert mo["eigvmax"] == mg["eigvmax"] and mo["umax"] == mg["umax"]


def test_fullsize_forms_agree_and_conserve(big):
    """200 steps: the FP64 form stays within 1e-12 of the exact form; the
    integrated density changes only by boundary fluxes, identically (to
    1e-12) in the exact and FP64 forms and to 1e-8 in the mixed form."""
    c, t, Q0, dt = big
    out = {}
    for prec in ("fp64_exact", "fp64", "mixed"):
        s = Solver(t, c.physics, precision=prec)
        s.set_state(Q0)
        m0 = s.monitor()["mass"]
        s.rk_s5p3(dt, 200)
        m1 = s.monitor()
        out[prec] = (s.state()["Q"], m0, m1)
        s.close()
    ref = out["fp64_exact"][0]
    assert np.isfinite(ref).all()
    assert rel_l2(out["fp64"][0], ref) <= 1e-12
    assert rel_l2(out["mixed"][0], ref) <= 1e-6
    dm = {k: (v[2]["mass"] - v[1]) / v[1] for k, v in out.items()}
    assert abs(dm["fp64"] - dm["fp64_exact"]) <= 1e-12
    assert abs(dm["mixed"] - dm["fp64_exact"]) <= 1e-8
    assert math.isfinite(out["mixed"][2]["divbsum"])
