"""The oracle's operation-count build (libsddc_oracle_count.so): the same
source compiled as C++ with a double that counts +, -, *, / and square roots
on state-dependent quantities.  It must compute exactly what the plain oracle
computes (bit-equal states), and its count per DOF-stage of RK_S5P3 (the
reference's FP64 operations, mu = eta0 = 0) must not depend on the mesh size
beyond the boundary faces' share.  The exact counts of one small case are
pinned, so a change to the oracle's arithmetic shows up here."""
import numpy as np
import pytest

from oracle import sddc_oracle as so
from sddc_b200 import cases, host, mesh


def _case(nr, nt, N, seed=3):
    m = mesh.cylinder_ogrid(nr, nt)
    t = host.build_tables(m, N)
    ph = cases.cylinder_physics(ms=0.5, ma=2.0)
    Q0 = cases.freestream_state(ph, N, m.ncell, noise=1e-6, seed=seed)
    return m, t, ph, Q0, cases.cfl_dt(m, Q0, N)


def _step_counts(t, ph, Q0, dt):
    o = so.Oracle(t, ph, count=True, skip_ideal_viscous=True)
    o.set_state(Q0)
    o.op_counts(reset=True)
    o.rk_s5p3(dt, 1)
    return o, o.op_counts(reset=True)


def test_count_build_computes_the_oracle_bit_for_bit():
    m, t, ph, Q0, dt = _case(8, 16, 4)
    oc, c = _step_counts(t, ph, Q0, dt)
    op = so.Oracle(t, ph, skip_ideal_viscous=True)
    op.set_state(Q0)
    op.rk_s5p3(dt, 1)
    assert np.array_equal(oc.state()["Q"], op.state()["Q"])
    assert np.array_equal(oc.state()["resid"], op.state()["resid"])
    # the pinned counts of this case (128 cells, N = 4, one RK_S5P3 step)
    assert c == {"add": 5714501, "mul": 7997962, "div": 746240, "sqrt": 16325}


@pytest.mark.parametrize("N,lo,hi", [(4, 1390, 1420), (5, 1555, 1585)])
def test_count_per_dof_stage_is_size_independent(N, lo, hi):
    per = []
    for nr, nt in ((8, 16), (16, 32)):
        m, t, ph, Q0, dt = _case(nr, nt, N)
        _, c = _step_counts(t, ph, Q0, dt)
        per.append(sum(c.values()) / (m.ncell * N * N * 5))
    assert lo < per[0] < hi and lo < per[1] < hi, per
    assert abs(per[0] - per[1]) < 0.01 * per[1], per


def test_counts_need_the_count_build():
    m, t, ph, Q0, dt = _case(4, 8, 3)
    with pytest.raises(ValueError):
        so.Oracle(t, ph).op_counts()
    with pytest.raises(ValueError):
        so.Oracle(t, ph, tangent=True, count=True)
