"""Synthetic quadrilateral meshes in the reference's input formats.

The reference reads three text files (readGRIDinfo.f90):

* cell file, one line per cell: ``IC IV1 IV2 IV3 IV4 ICTYPE ICKEY``
  (READ_CELL_DATA, readGRIDinfo.f90:1-37);
* vertex file, one line per vertex: ``IV X Y`` (READ_VRT_DATA, :40-84);
* boundary file, one line per boundary face:
  ``IB IV1 IV2 IREGION IPATCH TYPE`` with TYPE one of INLE, OUTL, SYMP, WALL,
  CYCL, FREE (READ_BND_DATA, :233-290);
* with CURVE_WALL = 1, the 8-node file: eight lines ``X Y`` per cell in
  global cell order, corners 1-4 counter-clockwise then the mid-side nodes
  of edges 1-2, 2-3, 3-4, 4-1 (READ_VRT8_DATA, :86-117).

The reference ships no meshes, so the cases are generated here:

* ``cylinder_ogrid``: the O-grid annulus around an adiabatic cylinder of
  diameter 1 (r in [0.5, 20]) with geometric radial stretching, cells
  counter-clockwise, the seam sharing its vertices (a rotational seam cannot
  be expressed as a translation-only CYCL pair, connect_bdry.f90:281-298).
  The inner ring is WALL; the outer ring is INLE where the free stream enters
  (u_inf . n < 0) and OUTL elsewhere.  ``curved=True`` adds the 8-node cells
  whose circumferential edges are circular arcs (their mid-side nodes on the
  circle), the reference's CURVE_WALL = 1 geometry.
* ``periodic_box``: a uniform box with every outer face CYCL.
* ``channel_box``: a box with one boundary type per side and optionally
  perturbed interior vertices (curved metrics), to exercise every BCFLUX
  branch.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

BC_NAMES = ("INLE", "OUTL", "SYMP", "WALL", "CYCL", "FREE")
BC_CODE = {n: i for i, n in enumerate(BC_NAMES)}


@dataclasses.dataclass
class Mesh:
    """A single-block quadrilateral mesh.

    ``ivcell`` is IVCELL(NCELL,4) with 1-based vertex ids, ``bnd_v`` is
    IVGBOUN(NB,2) and ``bnd_type`` holds indices into ``BC_NAMES``.
    """

    xv: np.ndarray
    yv: np.ndarray
    ivcell: np.ndarray
    bnd_v: np.ndarray
    bnd_type: np.ndarray
    dxcycl: float = 1.0
    dycycl: float = 1.0
    name: str = "mesh"
    xxf_cell: np.ndarray | None = None  # (2,8,NCELL) Fortran order: 8-node cells (CURVE_WALL = 1)

    @property
    def curved(self) -> bool:
        return self.xxf_cell is not None

    @property
    def ncell(self) -> int:
        return int(self.ivcell.shape[0])

    @property
    def nvert(self) -> int:
        return int(self.xv.shape[0])

    def min_edge(self) -> float:
        """Shortest cell edge (the h of the CFL time step)."""
        iv = self.ivcell - 1
        h = np.inf
        for a, b in ((0, 1), (1, 2), (2, 3), (3, 0)):
            d = np.hypot(self.xv[iv[:, a]] - self.xv[iv[:, b]], self.yv[iv[:, a]] - self.yv[iv[:, b]])
            h = min(h, float(d.min()))
        return h

    # -- the reference's text formats -------------------------------------
    def write(self, directory: str, stem: str | None = None) -> dict:
        """Write cell, vertex and boundary files; returns their paths."""
        stem = stem or self.name
        os.makedirs(directory, exist_ok=True)
        paths = {k: os.path.join(directory, f"{stem}.{k}") for k in ("cel", "vrt", "bnd")}
        nc = self.ncell
        cel = np.column_stack([np.arange(1, nc + 1), self.ivcell, np.ones(nc, int), np.ones(nc, int)])
        np.savetxt(paths["cel"], cel, fmt="%d")
        with open(paths["vrt"], "w") as f:
            for i, (x, y) in enumerate(zip(self.xv, self.yv), 1):
                f.write(f"{i} {x:.17e} {y:.17e}\n")
        with open(paths["bnd"], "w") as f:
            for i, ((a, b), t) in enumerate(zip(self.bnd_v, self.bnd_type), 1):
                f.write(f"{i} {a} {b} 1 1 {BC_NAMES[t]}\n")
        if self.curved:
            paths["vrt8"] = os.path.join(directory, f"{stem}.vrt8")
            with open(paths["vrt8"], "w") as f:
                for c in range(nc):
                    for k in range(8):
                        f.write(f"{self.xxf_cell[0, k, c]:.17e} {self.xxf_cell[1, k, c]:.17e}\n")
        return paths

    @classmethod
    def read(cls, cel: str, vrt: str, bnd: str, dxcycl: float = 1.0, dycycl: float = 1.0,
             vrt8: str | None = None) -> "Mesh":
        c = np.loadtxt(cel, dtype=np.int64, ndmin=2)
        v = np.loadtxt(vrt, dtype=np.float64, ndmin=2)
        order = np.argsort(v[:, 0])
        v = v[order]
        bv, bt = [], []
        with open(bnd) as f:
            for line in f:
                parts = line.split()
                if len(parts) < 6:
                    continue
                bv.append((int(parts[1]), int(parts[2])))
                bt.append(BC_CODE[parts[5][:4].upper()])
        xx8 = None
        if vrt8 is not None:
            a = np.loadtxt(vrt8, dtype=np.float64, ndmin=2)  # (8*NCELL, 2)
            xx8 = np.asfortranarray(a.reshape(c.shape[0], 8, 2).transpose(2, 1, 0))
        return cls(
            xv=np.ascontiguousarray(v[:, 1]),
            yv=np.ascontiguousarray(v[:, 2]),
            ivcell=np.ascontiguousarray(c[:, 1:5].astype(np.int32)),
            bnd_v=np.asarray(bv, dtype=np.int32).reshape(-1, 2),
            bnd_type=np.asarray(bt, dtype=np.int32),
            dxcycl=dxcycl,
            dycycl=dycycl,
            name=os.path.splitext(os.path.basename(cel))[0],
            xxf_cell=xx8,
        )


def eight_node_cells(m: Mesh, mid=None) -> np.ndarray:
    """xxf_cell (2,8,NCELL): the corners of each cell and its mid-side nodes.
    ``mid(xa, ya, xb, yb)`` places the node between two corners (arrays over
    cells); the default is the straight midpoint, which makes the 8-node map
    equal the bilinear one."""
    iv = m.ivcell - 1
    X, Y = m.xv[iv], m.yv[iv]  # (NCELL, 4)
    xx = np.zeros((2, 8, m.ncell), order="F")
    xx[0, :4], xx[1, :4] = X.T, Y.T
    mid = mid or (lambda xa, ya, xb, yb: (0.5 * (xa + xb), 0.5 * (ya + yb)))
    for k, (a, b) in enumerate(((0, 1), (1, 2), (2, 3), (3, 0))):
        xx[0, 4 + k], xx[1, 4 + k] = mid(X[:, a], Y[:, a], X[:, b], Y[:, b])
    return xx


def radial_ratio(nr: int, ratio32: float = 1.08) -> float:
    """Geometric radial ratio that keeps the 32-cell grading under refinement.

    A 32-cell annulus from r=0.5 to r=20 at ratio 1.08 stretches its cells by
    1.08**31 ~ 10.9; refining to ``nr`` cells with the same total stretch
    uses ratio**(32/nr).  A literal 1.08 at nr=256 would make the first cell
    about 4e-9 thick.
    """
    return ratio32 ** (32.0 / nr)


def cylinder_ogrid(nr: int, nt: int, r0: float = 0.5, r1: float = 20.0, ratio: float | None = None,
                   uinf: float = 1.0, vinf: float = 0.0, curved: bool = False) -> Mesh:
    """O-grid around a cylinder of radius ``r0``; cells ordered ring by ring."""
    q = radial_ratio(nr) if ratio is None else ratio
    if abs(q - 1.0) < 1e-14:
        dr = np.full(nr, (r1 - r0) / nr)
    else:
        dr0 = (r1 - r0) * (q - 1.0) / (q ** nr - 1.0)
        dr = dr0 * q ** np.arange(nr)
    r = np.concatenate([[r0], r0 + np.cumsum(dr)])
    r[-1] = r1
    th = 2.0 * np.pi * np.arange(nt) / nt
    # vertex (i, j): circumferential i in [0, nt), radial j in [0, nr]
    R, T = np.meshgrid(r, th, indexing="ij")  # (nr+1, nt)
    xv = (R * np.cos(T)).ravel()
    yv = (R * np.sin(T)).ravel()

    def vid(i, j):
        return j * nt + (i % nt) + 1

    i = np.arange(nt)
    cells = []
    for j in range(nr):
        # counter-clockwise in (x, y): radial edge first, then along theta
        cells.append(np.stack([vid(i, j), vid(i, j + 1), vid(i + 1, j + 1), vid(i + 1, j)], axis=1))
    ivcell = np.concatenate(cells).astype(np.int32)
    bv, bt = [], []
    for k in range(nt):  # inner wall
        bv.append((vid(k, 0), vid(k + 1, 0)))
        bt.append(BC_CODE["WALL"])
    for k in range(nt):  # outer ring: inflow where the free stream enters
        tm = 2.0 * np.pi * (k + 0.5) / nt
        inflow = uinf * math.cos(tm) + vinf * math.sin(tm) < 0.0
        bv.append((vid(k, nr), vid(k + 1, nr)))
        bt.append(BC_CODE["INLE" if inflow else "OUTL"])
    m = Mesh(xv, yv, ivcell, np.asarray(bv, np.int32), np.asarray(bt, np.int32), name=f"cyl{nr}x{nt}")
    if curved:
        def arc_mid(xa, ya, xb, yb):
            # an edge between two vertices of one ring is the arc between
            # them; a radial edge is straight
            ra, rb = np.hypot(xa, ya), np.hypot(xb, yb)
            same = np.abs(ra - rb) <= 1e-12 * np.maximum(ra, rb)
            ta, tb = np.arctan2(ya, xa), np.arctan2(yb, xb)
            dt = np.angle(np.exp(1j * (tb - ta)))  # the short way round, across the seam too
            tm = ta + 0.5 * dt
            return (np.where(same, ra * np.cos(tm), 0.5 * (xa + xb)),
                    np.where(same, ra * np.sin(tm), 0.5 * (ya + yb)))
        m.xxf_cell = eight_node_cells(m, arc_mid)
        m.name = f"cyl{nr}x{nt}c"
    return m


def periodic_box(nx: int, ny: int, lx: float = 2.0 * np.pi, ly: float = 2.0 * np.pi) -> Mesh:
    """Uniform box on [0,lx] x [0,ly] with all outer faces CYCL."""
    m = _box(nx, ny, lx, ly, ("CYCL",) * 4, 0.0, 0)
    m.dxcycl, m.dycycl = lx, ly
    m.name = f"box{nx}x{ny}"
    return m


def channel_box(nx: int, ny: int, lx: float = 2.0, ly: float = 1.0,
                sides=("SYMP", "OUTL", "FREE", "INLE"), jitter: float = 0.0, seed: int = 0,
                wall_bottom: bool = False) -> Mesh:
    """Box with one boundary type per side (bottom, right, top, left).

    ``jitter`` moves interior vertices by up to that fraction of a cell so
    the bilinear metrics vary from cell to cell.
    """
    s = list(sides)
    if wall_bottom:
        s[0] = "WALL"
    return _box(nx, ny, lx, ly, tuple(s), jitter, seed)


def _box(nx, ny, lx, ly, sides, jitter, seed) -> Mesh:
    x = np.linspace(0.0, lx, nx + 1)
    y = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(x, y, indexing="ij")  # (nx+1, ny+1)
    if jitter:
        rng = np.random.default_rng(seed)
        dx, dy = lx / nx, ly / ny
        X[1:-1, 1:-1] += jitter * dx * rng.uniform(-1, 1, (nx - 1, ny - 1))
        Y[1:-1, 1:-1] += jitter * dy * rng.uniform(-1, 1, (nx - 1, ny - 1))
    xv = X.T.ravel()  # vertex id = j*(nx+1) + i + 1
    yv = Y.T.ravel()

    def vid(i, j):
        return j * (nx + 1) + i + 1

    i = np.arange(nx)
    cells = [np.stack([vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)], axis=1) for j in range(ny)]
    ivcell = np.concatenate(cells).astype(np.int32)
    bv, bt = [], []
    for k in range(nx):
        bv.append((vid(k, 0), vid(k + 1, 0)))
        bt.append(BC_CODE[sides[0]])
    for k in range(ny):
        bv.append((vid(nx, k), vid(nx, k + 1)))
        bt.append(BC_CODE[sides[1]])
    for k in range(nx):
        bv.append((vid(k + 1, ny), vid(k, ny)))
        bt.append(BC_CODE[sides[2]])
    for k in range(ny):
        bv.append((vid(0, k + 1), vid(0, k)))
        bt.append(BC_CODE[sides[3]])
    return Mesh(xv, yv, ivcell, np.asarray(bv, np.int32), np.asarray(bt, np.int32), name=f"chan{nx}x{ny}")
