"""The benchmark cases: meshes, physical parameters and seeded initial states.

The reference ships no input decks, so every case is generated:

* cylinder: ideal MHD (gamma = 5/3) past an adiabatic cylinder of diameter 1.
  Free stream rho = 1, u = (1, 0), p = rho u^2 / (gamma Ms^2) (sonic Mach Ms),
  B = (u sqrt(rho) / MA, 0) (Alfven Mach MA), psi = 0; the state is the free
  stream plus seeded uniform noise U(-a, a) on all nine conserved variables
  (numpy default_rng(seed)).  vismode = 1, ARTIV = 1, mu = eta0 = 0.
* Orszag-Tang: periodic [0, 2 pi]^2, rho = 25/(36 pi), p = 5/(12 pi),
  u = (-sin y, sin x), B = (-sin y, sin 2x)/sqrt(4 pi), psi = 0, plus seeded
  U(-1e-8, 1e-8) noise.

The reference has no CFL logic (dt is fixed in QUAD.INP, readinput.f90:24);
``cfl_dt`` fixes dt = CFL * h_min / (N * lambda_max(IC)) once per case, with
h_min the shortest cell edge and lambda_max the largest |u| + c_fast of the
initial state.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import mesh as meshmod

GAMMA = 5.0 / 3.0


@dataclasses.dataclass
class Physics:
    rinf: float = 1.0
    pinf: float = 1.0
    uinf: float = 1.0
    vinf: float = 0.0
    bxinf: float = 0.0
    byinf: float = 0.0
    vismode: int = 1
    artiv: int = 1
    mu: float = 0.0
    eta0: float = 0.0
    dxcycl: float = 1.0
    dycycl: float = 1.0


def cylinder_physics(ms: float = 1.5, ma: float = 2.0) -> Physics:
    rho, u = 1.0, 1.0
    p = rho * u * u / (GAMMA * ms * ms)
    bx = u * math.sqrt(rho) / ma
    return Physics(rinf=rho, pinf=p, uinf=u, vinf=0.0, bxinf=bx, byinf=0.0)


def conserved(rho, u, v, w, p, bx, by, bz, psi):
    """Conserved variables from primitive ones (SETINITIALCOND's formula,
    setinitialcond.f90:17-37)."""
    rho = np.asarray(rho, dtype=np.float64)
    e = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w) + 0.5 * (bx * bx + by * by + bz * bz) + 0.5 * psi * psi
    return np.stack(np.broadcast_arrays(rho, rho * u, rho * v, rho * w, e, bx, by, bz, psi))


def freestream_state(ph: Physics, N: int, ncell: int, noise: float = 1e-6, seed: int = 0) -> np.ndarray:
    q0 = conserved(ph.rinf, ph.uinf, ph.vinf, 0.0, ph.pinf, ph.bxinf, ph.byinf, 0.0, 0.0).reshape(9)
    Q = np.empty((9, N, N, ncell), order="F")
    Q[...] = q0[:, None, None, None]
    if noise:
        rng = np.random.default_rng(seed)
        Q += rng.uniform(-noise, noise, size=(ncell, N, N, 9)).transpose(3, 2, 1, 0)
    return Q


def orszag_tang_state(xxsolu: np.ndarray, noise: float = 1e-8, seed: int = 0) -> np.ndarray:
    x, y = xxsolu[0], xxsolu[1]
    rho = np.full_like(x, 25.0 / (36.0 * math.pi))
    p = 5.0 / (12.0 * math.pi)
    s4 = math.sqrt(4.0 * math.pi)
    Q = conserved(rho, -np.sin(y), np.sin(x), 0.0, p, -np.sin(y) / s4, np.sin(2.0 * x) / s4, 0.0, 0.0)
    Q = np.asfortranarray(Q)
    if noise:
        rng = np.random.default_rng(seed)
        Q += rng.uniform(-noise, noise, size=Q.shape[::-1]).T
    return Q


def max_wave_speed(Q: np.ndarray) -> float:
    """Largest |u| + fast magnetosonic speed (perpendicular bound) of a state."""
    rho = Q[0]
    u, v, w = Q[1] / rho, Q[2] / rho, Q[3] / rho
    b2 = Q[5] ** 2 + Q[6] ** 2 + Q[7] ** 2
    p = (GAMMA - 1.0) * (Q[4] - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * b2 - 0.5 * Q[8] ** 2)
    cf = np.sqrt(GAMMA * p / rho + b2 / rho)
    return float(np.max(np.sqrt(u * u + v * v + w * w) + cf))


def cfl_dt(mesh: "meshmod.Mesh", Q: np.ndarray, N: int, cfl: float = 0.3) -> float:
    return cfl * mesh.min_edge() / (N * max_wave_speed(Q))


@dataclasses.dataclass
class Case:
    name: str
    mesh: "meshmod.Mesh"
    N: int
    physics: Physics
    steps: int
    seed: int = 0
    noise: float = 1e-6
    kind: str = "cylinder"

    @property
    def dof(self) -> int:
        return self.mesh.ncell * self.N * self.N

    def initial_state(self, tables=None) -> np.ndarray:
        if self.kind == "orszag_tang":
            return orszag_tang_state(tables.xxsolu, noise=self.noise, seed=self.seed)
        return freestream_state(self.physics, self.N, self.mesh.ncell, noise=self.noise, seed=self.seed)


def cylinder_case(nr: int, nt: int, N: int, steps: int = 500, ms: float = 1.5, ma: float = 2.0,
                  seed: int = 0, noise: float = 1e-6, curved: bool = False) -> Case:
    m = meshmod.cylinder_ogrid(nr, nt, curved=curved)
    return Case(name=f"cylinder_{nr}x{nt}_p{N - 1}", mesh=m, N=N, physics=cylinder_physics(ms, ma),
                steps=steps, seed=seed, noise=noise)


def orszag_tang_case(n: int, N: int = 4, steps: int = 100, seed: int = 0) -> Case:
    m = meshmod.periodic_box(n, n)
    ph = Physics(rinf=25.0 / (36.0 * math.pi), pinf=5.0 / (12.0 * math.pi), uinf=0.0, vinf=0.0,
                 dxcycl=2.0 * math.pi, dycycl=2.0 * math.pi)
    return Case(name=f"orszag_tang_{n}x{n}_p{N - 1}", mesh=m, N=N, physics=ph, steps=steps, seed=seed,
                noise=1e-8, kind="orszag_tang")


# the configurations the benchmark and the tests use
def config1(steps: int = 500) -> Case:
    """Cylinder 32 radial x 64 circumferential, p = 3, 500 RK3 steps."""
    return cylinder_case(32, 64, 4, steps)


def config2(steps: int = 2000) -> Case:
    """Cylinder 256 x 512, p = 4 (~3.3M solution points), 2000 RK3 steps."""
    return cylinder_case(256, 512, 5, steps)


def config3(n: int = 1024, steps: int = 100) -> Case:
    """Orszag-Tang 1024^2, p = 3."""
    return orszag_tang_case(n, 4, steps)
