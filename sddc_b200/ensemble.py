"""Batched ensembles: many independent cylinder cases in one launch per stage.

``make_cases`` draws the ensemble of the configured benchmark: cylinder
O-grids with sizes uniform over {16x32, 32x64, 64x128, 128x256}
(radial x circumferential), p = 3, seeded.  The configured sonic Mach range
[0.8, 2.0] diverges in the reference algorithm (its artificial viscosity is
computed but applied with zero coefficients, getrusanov.f90:326,328): on the
32x64 O-grid Ms = 0.8 reaches non-positive pressure after 469 RK3 steps and
a non-finite state after 496, Ms = 1.0 after 12 and 16, Ms = 1.5 after 4 and
6 (tests/test_configured_mach.py on the oracle, tests/test_gpu_configured.py
on the GPU).  The free streams are therefore drawn with Ms in [0.2, 0.3] and
the configured Alfven Mach range [1.5, 5.0]; each case keeps its own CFL
time step.

``merge`` concatenates the cases' set-up tables (cells, faces and face lists
renumbered) so that one drop-in context holds the whole batch; ``Batch``
drives it through ``sddc_set_cases`` / ``sddc_rk_step_cases``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import cases as casemod
from . import host
from .solver import Solver

SIZES = ((16, 32), (32, 64), (64, 128), (128, 256))


def make_cases(n: int = 64, seed: int = 0, N: int = 4, ms=(0.2, 0.3), ma=(1.5, 5.0)):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nr, nt = SIZES[int(rng.integers(len(SIZES)))]
        c = casemod.cylinder_case(nr, nt, N, ms=float(rng.uniform(*ms)), ma=float(rng.uniform(*ma)),
                                  seed=seed * 1000 + k, noise=1e-6)
        out.append(c)
    return out


def merge(tables_list):
    """Concatenated set-up tables of several cases with the same N."""
    N = tables_list[0].N
    assert all(t.N == N for t in tables_list)
    cell_off = face_off = 0
    parts = {k: [] for k in ("S1", "S2", "Jac", "xx", "IF2C", "IF2V", "inter", "inl", "out", "wal", "symp",
                             "free", "cyc", "ivc")}
    first = []
    for t in tables_list:
        first.append(cell_off)
        parts["S1"].append(t.S1)
        parts["S2"].append(t.S2)
        parts["Jac"].append(t.Jac)
        parts["xx"].append(t.xxsolu)
        F = t.IF2C.copy()
        F[:, 0] += cell_off
        F[:, 1] = np.where(F[:, 1] > 0, F[:, 1] + cell_off, 0)
        parts["IF2C"].append(F)
        parts["IF2V"].append(t.IF2V)
        for key, arr in (("inter", t.ibfinter), ("inl", t.ibfinl), ("out", t.ibfout), ("wal", t.ibfwal),
                         ("symp", t.ibfsymp), ("free", t.ibfree)):
            parts[key].append(arr + face_off)
        parts["cyc"].append(t.cyc2fpair + face_off)
        parts["ivc"].append(t.ivcell)
        cell_off += t.ncell
        face_off += t.nface

    def cat(key, axis=-1):
        return np.asfortranarray(np.concatenate(parts[key], axis=axis))

    counts = {k: sum(t.counts[k] for t in tables_list) for k in tables_list[0].counts}
    merged = host.Tables(
        N=N, ncell=cell_off, Lmat=tables_list[0].Lmat, Mmat=tables_list[0].Mmat, Xs=tables_list[0].Xs,
        Xf=tables_list[0].Xf, S1=cat("S1"), S2=cat("S2"), Jac=cat("Jac"), xxsolu=cat("xx"),
        IF2C=cat("IF2C", 0), IF2V=cat("IF2V", 0), ibfinter=np.concatenate(parts["inter"]).astype(np.int32),
        ibfinl=np.concatenate(parts["inl"]).astype(np.int32), ibfout=np.concatenate(parts["out"]).astype(np.int32),
        ibfwal=np.concatenate(parts["wal"]).astype(np.int32), ibfsymp=np.concatenate(parts["symp"]).astype(np.int32),
        ibfree=np.concatenate(parts["free"]).astype(np.int32), cyc2fpair=cat("cyc", 0).astype(np.int32),
        ivcell=cat("ivc", 0), counts=counts, dxcycl=1.0, dycycl=1.0)
    return merged, first


@dataclasses.dataclass
class Member:
    case: "casemod.Case"
    tables: "host.Tables"
    Q0: np.ndarray
    dt: float
    first_cell: int = 0


class Batch:
    """All members stepped together by one context: one launch per stage,
    either one CTA per tile or (persistent=True) as many CTAs as are resident,
    each walking the tile table largest case first."""

    def __init__(self, members, precision="mixed", cells_per_cta=0, persistent=False):
        self.members = members
        merged, first = merge([m.tables for m in members])
        for m, f in zip(members, first):
            m.first_cell = f
        self.tables = merged
        self.solver = Solver(merged, members[0].case.physics, precision=precision, cells_per_cta=cells_per_cta)
        recs = []
        for m in members:
            ph = m.case.physics
            recs.append(dict(first_cell=m.first_cell, ncell=m.tables.ncell, dt=m.dt, rinf=ph.rinf, pinf=ph.pinf,
                             uinf=ph.uinf, vinf=ph.vinf, bxinf=ph.bxinf, byinf=ph.byinf))
        self.solver.set_cases(recs)
        if persistent:
            self.solver.set_persistent(True)
        self.Q0 = np.asfortranarray(np.concatenate([m.Q0 for m in members], axis=-1))

    @property
    def dof(self) -> int:
        return self.tables.ncell * self.tables.N ** 2

    def reset(self):
        self.solver.set_state(self.Q0)

    def step(self, nsteps=1):
        self.solver.step_cases(nsteps)

    def member_state(self, Q, k):
        m = self.members[k]
        return Q[..., m.first_cell:m.first_cell + m.tables.ncell]

    def close(self):
        self.solver.close()


def build_members(case_list):
    out = []
    for c in case_list:
        t = host.build_tables(c.mesh, c.N)
        Q0 = c.initial_state(t)
        out.append(Member(case=c, tables=t, Q0=Q0, dt=casemod.cfl_dt(c.mesh, Q0, c.N)))
    return out
