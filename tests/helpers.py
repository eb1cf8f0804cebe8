"""Small seeded cases shared by the CPU and GPU tests."""
from __future__ import annotations

import math

import numpy as np

from sddc_b200 import cases, host, mesh


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def channel_physics(vismode=1):
    """A subsonic free stream for the channel boxes (every BC type)."""
    return cases.Physics(rinf=1.0, pinf=1.0, uinf=0.4, vinf=0.1, bxinf=0.3, byinf=0.2, vismode=vismode, artiv=1)


def smooth_state(tables, ph, amp=0.05, seed=0):
    """Free stream plus smooth sine perturbations (nonzero gradients of every
    variable, including Bz and psi), plus tiny seeded noise."""
    x, y = tables.xxsolu[0], tables.xxsolu[1]
    rho = ph.rinf * (1 + amp * np.sin(1.3 * x + 0.7 * y))
    u = ph.uinf + amp * np.cos(0.9 * x - 1.1 * y)
    v = ph.vinf + amp * np.sin(0.5 * x + 1.7 * y)
    w = amp * np.cos(1.1 * x + 0.3 * y)
    p = ph.pinf * (1 + amp * np.cos(0.4 * x - 0.8 * y))
    bx = ph.bxinf + amp * np.sin(0.6 * y)
    by = ph.byinf + amp * np.cos(0.8 * x)
    bz = amp * np.sin(x + y)
    psi = 0.1 * amp * np.cos(x - y)
    Q = np.asfortranarray(cases.conserved(rho, u, v, w, p, bx, by, bz, psi))
    rng = np.random.default_rng(seed)
    Q += 1e-7 * rng.uniform(-1, 1, Q.shape)
    return Q


def case_cylinder(nr=6, nt=12, N=4, seed=1):
    m = mesh.cylinder_ogrid(nr, nt)
    t = host.build_tables(m, N)
    ph = cases.cylinder_physics(ms=0.5, ma=2.0)
    Q = cases.freestream_state(ph, N, m.ncell, noise=1e-3, seed=seed)
    return m, t, ph, Q


def case_channel(nx=5, ny=4, N=4, sides=("SYMP", "OUTL", "FREE", "INLE"), jitter=0.2, vismode=1, seed=2):
    m = mesh.channel_box(nx, ny, sides=sides, jitter=jitter, seed=seed)
    t = host.build_tables(m, N)
    ph = channel_physics(vismode)
    Q = smooth_state(t, ph, seed=seed)
    return m, t, ph, Q


def case_periodic(n=5, N=4, seed=3):
    m = mesh.periodic_box(n, n + 1)
    t = host.build_tables(m, N)
    ph = cases.Physics(rinf=1.0, pinf=1.0, uinf=0.3, vinf=-0.2, bxinf=0.4, byinf=0.1, dxcycl=2 * math.pi,
                       dycycl=2 * math.pi)
    Q = smooth_state(t, ph, seed=seed)
    return m, t, ph, Q


def case_wall_box(nx=4, ny=4, N=4, vismode=1, seed=4):
    return case_channel(nx, ny, N, sides=("WALL", "OUTL", "SYMP", "INLE"), jitter=0.15, vismode=vismode, seed=seed)


def wavy_periodic_box(n=6, amp=0.08):
    """A periodic box of 8-node cells whose edges bulge by a periodic
    sine (shared and periodic partner edges get the same mid-side node)."""
    m = mesh.periodic_box(n, n)
    L = 2 * math.pi
    h = L / n

    def mid(xa, ya, xb, yb):
        mx, my = 0.5 * (xa + xb), 0.5 * (ya + yb)
        d = amp * h * np.sin(2 * math.pi * mx / L) * np.sin(2 * math.pi * my / L)
        return mx + d, my - d

    m.xxf_cell = mesh.eight_node_cells(m, mid)
    m.name = f"wavy{n}x{n}"
    return m


def case_cylinder_curved(nr=6, nt=12, N=4, seed=5):
    """The O-grid with 8-node cells (arcs for the circumferential edges)."""
    m = mesh.cylinder_ogrid(nr, nt, curved=True)
    t = host.build_tables(m, N)
    ph = cases.cylinder_physics(ms=0.5, ma=2.0)
    Q = cases.freestream_state(ph, N, m.ncell, noise=1e-3, seed=seed)
    return m, t, ph, Q


def case_wavy(n=5, N=5, seed=6):
    m = wavy_periodic_box(n)
    t = host.build_tables(m, N)
    ph = cases.Physics(rinf=1.0, pinf=1.0, uinf=0.3, vinf=-0.2, bxinf=0.4, byinf=0.1, dxcycl=2 * math.pi,
                       dycycl=2 * math.pi)
    Q = smooth_state(t, ph, seed=seed)
    return m, t, ph, Q


ALL_SMALL = {
    "cylinder_n4": lambda: case_cylinder(N=4),
    "cylinder_n5": lambda: case_cylinder(N=5),
    "channel_n3": lambda: case_channel(N=3),
    "channel_n4": lambda: case_channel(N=4),
    "channel_n5": lambda: case_channel(N=5),
    "periodic_n4": lambda: case_periodic(N=4),
    "wallbox_vis1": lambda: case_wall_box(vismode=1),
    "wallbox_vis0": lambda: case_wall_box(vismode=0),
    "periodic_n2": lambda: case_periodic(N=2),
    "cylinder_n6": lambda: case_cylinder(N=6),
    "cylinder_curved_n4": lambda: case_cylinder_curved(N=4),
    "wavybox_n5": lambda: case_wavy(N=5),
}
