"""The reference's run deck and restart file.

``QUAD.INP`` is read positionally by readinput (readinput.f90:6-44): every
line is a value except the separator lines the reader skips.  The restart
file is the unformatted stream written by WRITE_ALL_DATA_PARALLEL
(write_data.f90:5-83) and read by READ_ALL_DATA_BINARY
(read_data_restart.f90:35-67): int32 iter, float64 ctime, then per cell an
int32 global cell id followed by Q(9,N,N) in column-major order.  The seeded
initial states of the benchmark cases enter the reference through this file
(restart=1, restart_ord=N).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Deck:
    namecel: str = "grid.cel"
    namevrt: str = "grid.vrt"
    namevrt8: str = "grid.vrt8"
    namebnd: str = "grid.bnd"
    metis_cell: str = "grid.metis"
    namerestart: str = "restart.dat"
    N: int = 4
    curve_wall: int = 0
    vismode: int = 1
    mu: float = 0.0
    eta0: float = 0.0
    k_stage: int = 3
    dt: float = 1e-3
    maxiter: int = 100
    dxcycl: float = 1.0
    dycycl: float = 1.0
    artiv: int = 1
    nre: int = 1
    nwrite: int = 1000
    restart: int = 1
    restart_ord: int = 4
    rinf: float = 1.0
    pinf: float = 1.0
    uinf: float = 1.0
    vinf: float = 0.0
    bxinf: float = 0.0
    byinf: float = 0.0

    # (field, separator-before) in readinput order
    _LAYOUT = (
        ("#", "#"), ("namecel", None), ("namevrt", None), ("namevrt8", None), ("namebnd", None),
        ("metis_cell", None), ("namerestart", None), ("#", None), ("N", None), ("curve_wall", None),
        ("vismode", None), ("mu", None), ("eta0", None), ("#", None), ("k_stage", None), ("dt", None),
        ("maxiter", None), ("#", None), ("dxcycl", None), ("dycycl", None), ("#", None), ("artiv", None),
        ("#", None), ("nre", None), ("nwrite", None), ("#", None), ("restart", None),
        ("restart_ord", None), ("#", None), ("rinf", None), ("pinf", None), ("uinf", None),
        ("vinf", None), ("bxinf", None), ("byinf", None),
    )

    def write(self, path: str) -> None:
        lines = []
        for name, _ in self._LAYOUT:
            if name == "#":
                lines.append("# ----")
                continue
            v = getattr(self, name)
            if isinstance(v, float):
                lines.append(f"{v!r}")
            elif isinstance(v, str):
                lines.append(f"'{v}'")
            else:
                lines.append(str(v))
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")

    @classmethod
    def read(cls, path: str) -> "Deck":
        with open(path) as f:
            raw = [ln.rstrip("\n") for ln in f]
        d = cls()
        fields = {fl.name: fl.type for fl in dataclasses.fields(cls)}
        for (name, _), line in zip(cls._LAYOUT, raw):
            if name == "#":
                continue
            tok = line.split()[0].strip("'\"")
            typ = fields[name]
            if typ in ("int", int):
                val = int(tok)
            elif typ in ("float", float):
                val = float(tok.replace("d", "e").replace("D", "e"))
            else:
                val = tok
            setattr(d, name, val)
        return d


def write_restart(path: str, Q: np.ndarray, iter_: int = 0, ctime: float = 0.0) -> None:
    """Q has the Fortran shape (9,N,N,NCELL); cells are written in order."""
    nv, n, n2, nc = Q.shape
    assert nv == 9 and n == n2
    rec = np.dtype([("icg", "<i4"), ("q", "<f8", (nv * n * n,))])
    body = np.zeros(nc, dtype=rec)
    body["icg"] = np.arange(1, nc + 1, dtype=np.int32)
    body["q"] = np.asfortranarray(Q).reshape(nv * n * n, nc, order="F").T
    with open(path, "wb") as f:
        f.write(np.int32(iter_).tobytes())
        f.write(np.float64(ctime).tobytes())
        f.write(body.tobytes())


def read_restart(path: str, N: int, ncell: int):
    """Returns (Q (9,N,N,NCELL) Fortran order, iter, ctime)."""
    with open(path, "rb") as f:
        it = int(np.frombuffer(f.read(4), "<i4")[0])
        ct = float(np.frombuffer(f.read(8), "<f8")[0])
        rec = np.dtype([("icg", "<i4"), ("q", "<f8", (9 * N * N,))])
        body = np.frombuffer(f.read(rec.itemsize * ncell), dtype=rec)
    Q = np.zeros((9, N, N, ncell), order="F")
    flat = Q.reshape(9 * N * N, ncell, order="F")
    flat[:, body["icg"] - 1] = body["q"].T
    return Q, it, ct
