"""The viscous / resistive chain (vismode = 1, mu and eta0 > 0) against the
CPU oracle's full chain (nablaQsp, interior and face gradient averaging,
BCVISFLUX with the adiabatic-wall energy gradient, comp_viscous_flux), through
the C ABI.  Bars as for the ideal chain: the exact FP64 form bit-exact, the
FP64 form within 1e-12 relative after a step, the mixed form within 1e-6."""
import dataclasses

import numpy as np
import pytest

import sddc_oracle as O
from helpers import ALL_SMALL, rel_l2
from sddc_b200 import cases
from sddc_b200.solver import SddcError, Solver

pytestmark = pytest.mark.gpu

# every boundary kind (channel: SYMP, OUTL, FREE, INLE; wall box: WALL),
# cyclic pairs (periodic) and the O-grid's curved walls; N = 3, 4, 5
VISC_CASES = ["cylinder_n4", "channel_n3", "channel_n5", "periodic_n4", "wallbox_vis1"]


def _viscous(name, mu=0.02, eta0=0.015):
    m, t, ph, Q = ALL_SMALL[name]()
    ph = dataclasses.replace(ph, mu=mu, eta0=eta0, vismode=1)
    return m, t, ph, Q


@pytest.mark.parametrize("name", VISC_CASES)
def test_viscous_compresid_exact(name):
    m, t, ph, Q = _viscous(name)
    o = O.Oracle(t, ph)
    s = Solver(t, ph, precision="fp64_exact")
    o.set_state(Q)
    s.set_state(Q)
    for _ in range(2):
        o.compresid()
        s.compresid()
        a, g = o.state(), s.state(resid=True, nablaQs=True)
        assert np.array_equal(g["resid"], a["resid"]), rel_l2(g["resid"], a["resid"])
        assert np.array_equal(g["nablaQs"], a["nablaQs"])
    # the viscous part is not negligible in these cases
    oi = O.Oracle(t, dataclasses.replace(ph, mu=0.0, eta0=0.0))
    oi.set_state(Q)
    oi.compresid()
    oi.compresid()
    assert rel_l2(oi.state()["resid"], a["resid"]) > 1e-4
    s.close()


@pytest.mark.parametrize("name", VISC_CASES)
@pytest.mark.parametrize("k_stage", [3, 5])
def test_viscous_rk_exact(name, k_stage):
    m, t, ph, Q = _viscous(name)
    dt = 0.2 * cases.cfl_dt(m, Q, t.N)
    o = O.Oracle(t, ph)
    s = Solver(t, ph, precision="fp64_exact", k_stage=k_stage)
    o.set_state(Q)
    s.set_state(Q)
    if k_stage == 3:
        o.rk_s5p3(dt, 4)
        s.rk_s5p3(dt, 4)
    else:
        o.five_stage_rk(dt, 3)
        s.rk_s5p3(dt, 3)  # the context's k_stage selects FiveStageRk
    assert np.array_equal(s.state()["Q"], o.state()["Q"])
    s.close()


@pytest.mark.parametrize("name", ["cylinder_n4", "wallbox_vis1", "periodic_n4"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_viscous_forms(name, precision, tol):
    m, t, ph, Q = _viscous(name)
    dt = 0.2 * cases.cfl_dt(m, Q, t.N)
    o = O.Oracle(t, ph)
    s = Solver(t, ph, precision=precision)
    o.set_state(Q)
    s.set_state(Q)
    o.rk_s5p3(dt, 1)
    s.rk_s5p3(dt, 1)
    assert rel_l2(s.state()["Q"], o.state()["Q"]) <= tol
    s.close()


def test_viscous_rejections():
    m, t, ph, Q = _viscous("cylinder_n4")
    s = Solver(t, ph, precision="fp64_exact")
    with pytest.raises(SddcError):
        s.set_cases([dict(first_cell=0, ncell=t.ncell, dt=1e-3, rinf=ph.rinf, pinf=ph.pinf, uinf=ph.uinf,
                          vinf=ph.vinf, bxinf=ph.bxinf, byinf=ph.byinf)])
    s.set_state(Q)
    with pytest.raises(SddcError):
        s.adjoint_run(1e-3, 2, 0, 2)
    s.close()
    with pytest.raises(SddcError):
        Solver(t, dataclasses.replace(ph, mu=-1.0), precision="fp64")
