"""The configured cylinder Mach numbers under the reference's algorithm.

The cylinder configurations name sonic Mach 1.5 (the single cases) and
Ms in [0.8, 2.0] (the ensemble).  The reference computes an artificial
viscosity but its coefficients are hard-coded to zero (getrusanov.f90:326,
328), and nothing else limits the high-order solution at the bow shock of
the impulsive start: with the configured free stream the oracle (the FP64
restatement of the reference's path) reaches non-positive pressure within a
few RK3 steps and non-finite values soon after.  These tests pin that on the
configured 32 x 64, p = 3 O-grid at CFL 0.3, and pin that the Ms = 0.5 case
the benchmarks run instead stays positive.  The GPU side of the same window
(bit-equal to the oracle up to the fault, and the device's fault report) is
in tests/test_gpu_orszag_tang.py.
"""
import numpy as np
import pytest

import sddc_oracle as O
from sddc_b200 import cases, host

GAMMA = 5.0 / 3.0


def pressure(Q):
    rho = Q[0]
    ke = 0.5 * (Q[1] ** 2 + Q[2] ** 2 + Q[3] ** 2) / rho
    return (GAMMA - 1.0) * (Q[4] - ke - 0.5 * (Q[5] ** 2 + Q[6] ** 2 + Q[7] ** 2) - 0.5 * Q[8] ** 2)


def run_until_fault(ms, max_steps):
    """RK3 steps of the configured 32 x 64, p = 3 cylinder (MA = 2, seeded
    1e-6 noise, CFL 0.3) on the oracle: the first step after which some
    pressure or density is <= 0, and the first after which a value is not
    finite (None: not within max_steps)."""
    c = cases.cylinder_case(32, 64, 4, ms=ms, ma=2.0)
    t = host.build_tables(c.mesh, c.N)
    Q0 = c.initial_state(t)
    dt = cases.cfl_dt(c.mesh, Q0, c.N, 0.3)
    o = O.Oracle(t, c.physics)
    o.set_state(Q0)
    first_nonpos = first_nonfinite = None
    for step in range(1, max_steps + 1):
        o.rk_s5p3(dt, 1)
        Q = o.state()["Q"]
        if not np.isfinite(Q).all():
            first_nonfinite = step
            break
        if first_nonpos is None and (pressure(Q).min() <= 0.0 or Q[0].min() <= 0.0):
            first_nonpos = step
    return first_nonpos, first_nonfinite


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(8)


@pytest.mark.parametrize("ms,nonpos,nonfinite", [(1.5, 4, 6), (1.0, 12, 16)])
def test_configured_supersonic_inflow_diverges(ms, nonpos, nonfinite):
    """Ms = 1.5 (configs 1, 2 and 5) and Ms = 1.0: negative pressure after
    4 (12) steps, non-finite state after 6 (16)."""
    assert run_until_fault(ms, 40) == (nonpos, nonfinite)


def test_benchmarked_mach_stays_positive():
    """Ms = 0.5, the Mach number the benchmarks run: positive pressure and
    density over the first 40 steps (500 steps are checked on the GPU
    against the oracle in test_gpu_parity.test_config1_500_steps)."""
    assert run_until_fault(0.5, 40) == (None, None)
