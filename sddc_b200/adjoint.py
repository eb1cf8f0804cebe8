"""Gradients of time-averaged cylinder drag and lift through the discrete
adjoint (``sddc_adjoint_run`` of the C ABI), and the torch.autograd.Function
that wraps it.

The objective is J = mean over the states after n1..n2 RK_S5P3 steps of
w_drag*C_D + w_lift*C_L, with C = 2F/(rho_inf |U_inf|^2 D) and F the force on
the wall faces (the momentum components of their Rusanov flux).  Its inputs
are the initial conserved field Q0 and the free stream (rinf, pinf, uinf,
vinf, bxinf, byinf) that the boundary states read; the time step is held
fixed.  The inflow sonic and Alfven Mach numbers enter through the free
stream (p = rho u^2/(gamma Ms^2), Bx = u sqrt(rho)/MA) and, when the caller
builds Q0 from them, through Q0 as well: ``DragLift`` is differentiable in
both, so autograd composes the two paths.

There is no CPU path: the product runs on the GPU through libsddc_b200.so.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import cases
from .solver import Solver

FREESTREAM = ("rinf", "pinf", "uinf", "vinf", "bxinf", "byinf")


def cylinder_freestream(ms, ma, rho: float = 1.0, u: float = 1.0):
    """The cylinder free stream as a differentiable function of the sonic and
    Alfven Mach numbers (torch tensors or floats): the 6-vector (rinf, pinf,
    uinf, vinf, bxinf, byinf) of cases.cylinder_physics."""
    ms = torch.as_tensor(ms, dtype=torch.float64)
    ma = torch.as_tensor(ma, dtype=torch.float64)
    p = rho * u * u / (cases.GAMMA * ms * ms)
    bx = u * math.sqrt(rho) / ma
    z = torch.zeros((), dtype=torch.float64)
    return torch.stack([z + rho, p, z + u, z, bx, z])


def freestream_field(fs, N: int, ncell: int, noise=None):
    """Q0 = the free stream fs (a torch 6-vector) at every solution point,
    plus an optional fixed noise array (9, N, N, ncell); differentiable in
    fs (conserved variables as SETINITIALCOND forms them)."""
    rho, p, u, v, bx, by = fs[0], fs[1], fs[2], fs[3], fs[4], fs[5]
    e = p / (cases.GAMMA - 1.0) + 0.5 * rho * (u * u + v * v) + 0.5 * (bx * bx + by * by)
    z = torch.zeros((), dtype=torch.float64)
    q = torch.stack([rho, rho * u, rho * v, z, e, bx, by, z, z])
    Q = q.reshape(9, 1, 1, 1).expand(9, N, N, ncell)
    if noise is not None:
        Q = Q + torch.as_tensor(noise, dtype=torch.float64)
    return Q


class DragLiftProblem:
    """The objective's fixed data: mesh tables, time step, step count,
    window and weights.  One GPU context per free stream is kept (the free
    stream is a creation parameter of the drop-in)."""

    def __init__(self, tables, dt: float, nsteps: int, n1: int, n2: int, w_drag: float = 1.0, w_lift: float = 0.0,
                 diameter: float = 1.0, checkpoint_every: int = 20, vismode: int = 1, artiv: int = 1,
                 cells_per_cta: int = 0):
        self.tables = tables
        self.dt, self.nsteps, self.n1, self.n2 = float(dt), int(nsteps), int(n1), int(n2)
        self.w_drag, self.w_lift, self.diameter = float(w_drag), float(w_lift), float(diameter)
        self.checkpoint_every = int(checkpoint_every)
        self.vismode, self.artiv = vismode, artiv
        self.cells_per_cta = int(cells_per_cta)
        self._solvers = {}
        self.last = None

    def solver(self, fs) -> Solver:
        key = tuple(float(x) for x in fs)
        s = self._solvers.get(key)
        if s is None:
            ph = cases.Physics(**dict(zip(FREESTREAM, key)), vismode=self.vismode, artiv=self.artiv)
            s = Solver(self.tables, ph, precision="fp64_exact", cells_per_cta=self.cells_per_cta)
            self._solvers[key] = s
        return s

    def run(self, Q0: np.ndarray, fs, gradient: bool = True) -> dict:
        """J (and dJ/dQ0, dJ/dfs) for the initial field Q0 and free stream fs."""
        s = self.solver(fs)
        s.set_state(np.asfortranarray(Q0, dtype=np.float64))
        r = s.adjoint_run(self.dt, self.nsteps, self.n1, self.n2, w_drag=self.w_drag, w_lift=self.w_lift,
                          diameter=self.diameter, checkpoint_every=self.checkpoint_every, gradient=gradient)
        self.last = r
        return r

    def close(self):
        for s in self._solvers.values():
            s.close()
        self._solvers.clear()


class DragLift(torch.autograd.Function):
    """J(Q0, fs) for a DragLiftProblem, with the discrete adjoint as its
    backward.  Q0: (9, N, N, ncell) float64 tensor; fs: 6-vector tensor."""

    @staticmethod
    def forward(ctx, Q0, fs, problem):
        r = problem.run(Q0.detach().cpu().numpy(), fs.detach().cpu().numpy(), gradient=True)
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(r["Qbar0"])), torch.from_numpy(r["parbar"]))
        return torch.tensor(r["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        qbar, pbar = ctx.saved_tensors
        return gJ * qbar, gJ * pbar, None


def mach_gradients(problem: DragLiftProblem, ms: float, ma: float, noise=None):
    """J and its total derivatives with respect to the inflow sonic and
    Alfven Mach numbers of a cylinder case whose initial field is the free
    stream (plus the fixed noise): both the boundary states and Q0 depend on
    them.  Returns (J, dJ/dMs, dJ/dMA, dJ/dQ0)."""
    ms_t = torch.tensor(float(ms), dtype=torch.float64, requires_grad=True)
    ma_t = torch.tensor(float(ma), dtype=torch.float64, requires_grad=True)
    fs = cylinder_freestream(ms_t, ma_t)
    t = problem.tables
    Q0 = freestream_field(fs, t.N, t.ncell, noise)
    J = DragLift.apply(Q0, fs, problem)
    J.backward()
    return float(J.detach()), float(ms_t.grad), float(ma_t.grad), problem.last["Qbar0"]
