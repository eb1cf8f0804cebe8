"""Batched ensembles: one context, one launch per stage over all cases, equal
bit for bit to running each case on its own context."""
import numpy as np
import pytest

import sddc_oracle as O
from sddc_b200 import cases, ensemble
from sddc_b200.solver import Solver

def _members():
    cl = [cases.cylinder_case(6, 12, 4, ms=0.25, ma=2.0, seed=1, noise=1e-4),
          cases.cylinder_case(4, 16, 4, ms=0.3, ma=4.0, seed=2, noise=1e-4),
          cases.cylinder_case(9, 10, 4, ms=0.2, ma=1.5, seed=3, noise=1e-4)]
    return ensemble.build_members(cl)


def _large_members():
    """More tiles than CTAs are resident at once, so that persistent CTAs
    walk several tiles; one case size not a multiple of the tile."""
    cl = [cases.cylinder_case(64, 128, 4, ms=0.25, ma=2.0, seed=4, noise=1e-4),
          cases.cylinder_case(9, 10, 4, ms=0.3, ma=4.0, seed=5, noise=1e-4),
          cases.cylinder_case(60, 100, 4, ms=0.2, ma=1.5, seed=6, noise=1e-4),
          cases.cylinder_case(48, 96, 4, ms=0.22, ma=3.0, seed=7, noise=1e-4)]
    return ensemble.build_members(cl)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "mixed"])
@pytest.mark.parametrize("cpb", [4, 6, 8])
@pytest.mark.parametrize("persistent", [False, True])
def test_batch_equals_separate_runs(precision, cpb, persistent):
    members = _members() if not persistent else _large_members()
    b = ensemble.Batch(members, precision=precision, cells_per_cta=cpb, persistent=persistent)
    b.reset()
    b.step(3)
    Qb = b.solver.state()["Q"]
    for k, m in enumerate(members):
        s = Solver(m.tables, m.case.physics, precision=precision, cells_per_cta=cpb)
        s.set_state(m.Q0)
        s.rk_s5p3(m.dt, 3)
        assert np.array_equal(b.member_state(Qb, k), s.state()["Q"])
        mx = s.maxima()
        assert b.solver.case_maxima(k) == (mx["eigvmax"], mx["umax"])
        s.close()
    b.close()


@pytest.mark.gpu
def test_batch_exact_equals_oracle():
    members = _members()
    b = ensemble.Batch(members, precision="fp64_exact")
    b.reset()
    b.step(2)
    Qb = b.solver.state()["Q"]
    for k, m in enumerate(members):
        o = O.Oracle(m.tables, m.case.physics)
        o.set_state(m.Q0)
        o.rk_s5p3(m.dt, 2)
        assert np.array_equal(b.member_state(Qb, k), o.state()["Q"])
    b.close()


def test_ensemble_generator_and_merge():
    cl = ensemble.make_cases(6, seed=5)
    assert all(c.N == 4 for c in cl)
    ms = [1.0 / np.sqrt(cases.GAMMA * c.physics.pinf) for c in cl]  # rho = u = 1
    assert all(0.2 - 1e-12 <= m <= 0.3 + 1e-12 for m in ms)
    members = ensemble.build_members(cl)
    merged, first = ensemble.merge([m.tables for m in members])
    assert merged.ncell == sum(m.tables.ncell for m in members)
    assert first[0] == 0 and all(first[i + 1] - first[i] == members[i].tables.ncell for i in range(5))
    assert merged.IF2C[:, 0].max() <= merged.ncell and merged.IF2C[:, 1].max() <= merged.ncell
