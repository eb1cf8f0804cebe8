"""Host-side set-up through libsddc_host.so (include/sddc_host.h).

``build_tables(mesh, N)`` runs the single-rank equivalent of the reference
host's set-up sequence (main.f90:22-52: CHECK_MESH, CONNECTIVITY,
CONNECT_BDRY, MAPCYCLOC, INIT_SETUP's operators and calcjacob) and returns
every array the residual drop-in takes, in the reference's Fortran layout
(column-major numpy arrays, 1-based index tables).
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _native
from ._native import ptr

_I = ctypes.c_int
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)

MC_FIELDS = ("nface", "ninter", "ninlet", "noutlet", "nsymp", "nwall", "ncycl", "ncycloc", "ncycrem",
             "npair", "nprocint", "nfree", "nreversed", "nvert", "ncell")


def _lib():
    lib = _native.load(_native.HOST_LIB)
    if not getattr(lib, "_sddc_typed", False):
        lib.sddc_sd_operators.argtypes = [_I, _PD, _PD, _PD, _PD]
        lib.sddc_mesh_build.argtypes = [ctypes.POINTER(ctypes.c_void_p), _I, _I, _PI, _PD, _PD, _I, _PI, _PI,
                                        _D, _D]
        lib.sddc_mesh_destroy.argtypes = [ctypes.c_void_p]
        lib.sddc_mesh_destroy.restype = None
        lib.sddc_mesh_counts.argtypes = [ctypes.c_void_p, _PI]
        lib.sddc_mesh_tables.argtypes = [ctypes.c_void_p] + [_PI] * 10
        lib.sddc_mesh_metrics.argtypes = [ctypes.c_void_p, _I, _PD, _PD, _PD, _PD]
        lib.sddc_metrics8.argtypes = [_I, _I, _PD, _PD, _PD, _PD, _PD]
        lib.sddc_plotmesh_build.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, _I, _PD]
        lib.sddc_plotmesh_destroy.argtypes = [ctypes.c_void_p]
        lib.sddc_plotmesh_destroy.restype = None
        lib.sddc_plotmesh_counts.argtypes = [ctypes.c_void_p, _PI, _PI]
        lib.sddc_plotmesh_tables.argtypes = [ctypes.c_void_p, _PD, _PI, _PI, _PI]
        lib.sddc_restart_filename.argtypes = [_I, ctypes.c_char_p, _I]
        lib.sddc_tecplot_filename.argtypes = [_D, ctypes.c_char_p, _I]
        lib.sddc_restart_write.argtypes = [ctypes.c_char_p, _I, _D, _I, _I, _PI, _PD]
        lib.sddc_restart_read.argtypes = [ctypes.c_char_p, _I, _I, _I, _PI, _I, _PD, _PI, _PD]
        lib.sddc_tecplot_write.argtypes = [ctypes.c_char_p, _D, _I, _I, _PD, _PD, _PD, _PI]
        lib.sddc_host_last_error.restype = ctypes.c_char_p
        lib._sddc_typed = True
    return lib


class HostError(RuntimeError):
    pass


def _check(rc: int, lib) -> None:
    if rc != 0:
        raise HostError(f"sddc host error {rc}: {lib.sddc_host_last_error().decode()}")


def sd_operators(N: int):
    """(Xs, Xf, Lmat, Mmat) with Lmat, Mmat shaped (N+1, N), Fortran order."""
    lib = _lib()
    Xs = np.zeros(N)
    Xf = np.zeros(N + 1)
    L = np.zeros((N + 1, N), order="F")
    M = np.zeros((N + 1, N), order="F")
    _check(lib.sddc_sd_operators(N, ptr(Xs), ptr(Xf), ptr(L), ptr(M)), lib)
    return Xs, Xf, L, M


@dataclasses.dataclass
class Tables:
    """Everything the drop-in needs besides the state, reference layout."""

    N: int
    ncell: int
    Lmat: np.ndarray
    Mmat: np.ndarray
    Xs: np.ndarray
    Xf: np.ndarray
    S1: np.ndarray      # (2,2,N+1,N,NCELL)
    S2: np.ndarray      # (2,2,N,N+1,NCELL)
    Jac: np.ndarray     # (N,N,NCELL)
    xxsolu: np.ndarray  # (2,N,N,NCELL)
    IF2C: np.ndarray    # (NFACE,4)
    IF2V: np.ndarray    # (NFACE,2)
    ibfinter: np.ndarray
    ibfinl: np.ndarray
    ibfout: np.ndarray
    ibfwal: np.ndarray
    ibfsymp: np.ndarray
    ibfree: np.ndarray
    cyc2fpair: np.ndarray  # (NPAIR,2)
    ivcell: np.ndarray     # (NCELL,4) after CHECK_MESH
    counts: dict
    dxcycl: float
    dycycl: float

    @property
    def nface(self) -> int:
        return int(self.IF2C.shape[0])

    def table_args(self):
        """Positional table arguments in sddc_set_tables order (numpy arrays and ints)."""
        return (self.Lmat, self.Mmat, self.S1, self.S2, self.Jac, self.IF2C, self.nface,
                self.ibfinter, len(self.ibfinter), self.ibfinl, len(self.ibfinl), self.ibfout,
                len(self.ibfout), self.ibfwal, len(self.ibfwal), self.ibfsymp, len(self.ibfsymp),
                self.ibfree, len(self.ibfree), self.cyc2fpair, int(self.cyc2fpair.shape[0]))


def _mesh_handle(lib, mesh) -> ctypes.c_void_p:
    iv = np.asfortranarray(mesh.ivcell.astype(np.int32))
    xv = np.ascontiguousarray(mesh.xv, dtype=np.float64)
    yv = np.ascontiguousarray(mesh.yv, dtype=np.float64)
    bv = np.asfortranarray(mesh.bnd_v.astype(np.int32).reshape(-1, 2))
    bt = np.ascontiguousarray(mesh.bnd_type.astype(np.int32))
    h = ctypes.c_void_p()
    _check(lib.sddc_mesh_build(ctypes.byref(h), mesh.ncell, mesh.nvert, ptr(iv, _I), ptr(xv), ptr(yv),
                               int(bt.shape[0]), ptr(bv, _I), ptr(bt, _I), float(mesh.dxcycl),
                               float(mesh.dycycl)), lib)
    return h


def build_tables(mesh, N: int) -> Tables:
    lib = _lib()
    h = _mesh_handle(lib, mesh)
    try:
        c = np.zeros(len(MC_FIELDS), dtype=np.int32)
        _check(lib.sddc_mesh_counts(h, ptr(c, _I)), lib)
        counts = dict(zip(MC_FIELDS, (int(x) for x in c)))
        nf, nc = counts["nface"], counts["ncell"]
        IF2C = np.zeros((nf, 4), np.int32, order="F")
        IF2V = np.zeros((nf, 2), np.int32, order="F")
        lists = {k: np.zeros(counts[n], np.int32) for k, n in
                 (("inter", "ninter"), ("inl", "ninlet"), ("out", "noutlet"), ("wal", "nwall"),
                  ("symp", "nsymp"), ("free", "nfree"))}
        cyc = np.zeros((counts["npair"], 2), np.int32, order="F")
        ivc = np.zeros((nc, 4), np.int32, order="F")
        _check(lib.sddc_mesh_tables(h, ptr(IF2C, _I), ptr(IF2V, _I), ptr(lists["inter"], _I),
                                    ptr(lists["inl"], _I), ptr(lists["out"], _I), ptr(lists["wal"], _I),
                                    ptr(lists["symp"], _I), ptr(lists["free"], _I), ptr(cyc, _I),
                                    ptr(ivc, _I)), lib)
        S1 = np.zeros((2, 2, N + 1, N, nc), order="F")
        S2 = np.zeros((2, 2, N, N + 1, nc), order="F")
        Jac = np.zeros((N, N, nc), order="F")
        xx = np.zeros((2, N, N, nc), order="F")
        if mesh.curved:  # CURVE_WALL = 1: the 8-node map
            x8 = np.asfortranarray(mesh.xxf_cell, dtype=np.float64)
            _check(lib.sddc_metrics8(N, nc, ptr(x8), ptr(S1), ptr(S2), ptr(Jac), ptr(xx)), lib)
        else:
            _check(lib.sddc_mesh_metrics(h, N, ptr(S1), ptr(S2), ptr(Jac), ptr(xx)), lib)
    finally:
        lib.sddc_mesh_destroy(h)
    Xs, Xf, L, M = sd_operators(N)
    return Tables(N=N, ncell=nc, Lmat=L, Mmat=M, Xs=Xs, Xf=Xf, S1=S1, S2=S2, Jac=Jac, xxsolu=xx, IF2C=IF2C,
                  IF2V=IF2V, ibfinter=lists["inter"], ibfinl=lists["inl"], ibfout=lists["out"],
                  ibfwal=lists["wal"], ibfsymp=lists["symp"], ibfree=lists["free"], cyc2fpair=cyc,
                  ivcell=ivc, counts=counts, dxcycl=float(mesh.dxcycl), dycycl=float(mesh.dycycl))


@dataclasses.dataclass
class PlotMesh:
    """The Tecplot plot mesh of tecplotter2dsetup (tecplotter2dsetup.f90:1-160), reference layout."""

    nre: int
    plotnodes: int
    plotcells: int
    plotx: np.ndarray         # (2,plotnodes)
    gnumnode: np.ndarray      # (nre+1,nre+1,NCELL), 1-based node numbers
    gnode_factor: np.ndarray  # (plotnodes)
    connec: np.ndarray        # (4,plotcells), 1-based


def plot_mesh(mesh, nre: int) -> PlotMesh:
    lib = _lib()
    h = _mesh_handle(lib, mesh)
    pm = ctypes.c_void_p()
    try:
        x8 = None if not mesh.curved else np.asfortranarray(mesh.xxf_cell, dtype=np.float64)
        _check(lib.sddc_plotmesh_build(ctypes.byref(pm), h, int(nre), ptr(x8)), lib)
        nn, nc = _I(), _I()
        _check(lib.sddc_plotmesh_counts(pm, ctypes.byref(nn), ctypes.byref(nc)), lib)
        px = np.zeros((2, nn.value), order="F")
        gn = np.zeros((nre + 1, nre + 1, mesh.ncell), np.int32, order="F")
        gf = np.zeros(nn.value, np.int32)
        cn = np.zeros((4, nc.value), np.int32, order="F")
        _check(lib.sddc_plotmesh_tables(pm, ptr(px), ptr(gn, _I), ptr(gf, _I), ptr(cn, _I)), lib)
    finally:
        if pm.value:
            lib.sddc_plotmesh_destroy(pm)
        lib.sddc_mesh_destroy(h)
    return PlotMesh(int(nre), nn.value, nc.value, px, gn, gf, cn)


def restart_filename(iter_: int) -> str:
    lib = _lib()
    b = ctypes.create_string_buffer(64)
    _check(0 if lib.sddc_restart_filename(int(iter_), b, 64) >= 0 else -1, lib)
    return b.value.decode()


def tecplot_filename(ctime: float) -> str:
    lib = _lib()
    b = ctypes.create_string_buffer(64)
    _check(0 if lib.sddc_tecplot_filename(float(ctime), b, 64) >= 0 else -1, lib)
    return b.value.decode()


def restart_write(path: str, Q: np.ndarray, iter_: int = 0, ctime: float = 0.0, icg=None) -> None:
    """WRITE_ALL_DATA_PARALLEL's file from a host Q (9,N,N,NCELL)."""
    lib = _lib()
    Q = np.asfortranarray(Q, dtype=np.float64)
    N, nc = Q.shape[1], Q.shape[3]
    g = None if icg is None else np.ascontiguousarray(icg, dtype=np.int32)
    _check(lib.sddc_restart_write(str(path).encode(), int(iter_), float(ctime), N, nc,
                                  None if g is None else ptr(g, _I), ptr(Q)), lib)


def restart_read(path: str, N: int, ncell: int, nrec: int = 0, icg2ic=None):
    """READ_ALL_DATA_BINARY: returns (Q (9,N,N,NCELL), iter, ctime); cells absent from the file stay 0."""
    lib = _lib()
    Q = np.zeros((9, N, N, ncell), order="F")
    m = None if icg2ic is None else np.ascontiguousarray(icg2ic, dtype=np.int32)
    it, ct = _I(), _D()
    _check(lib.sddc_restart_read(str(path).encode(), N, ncell, int(nrec), None if m is None else ptr(m, _I),
                                 0 if m is None else len(m), ptr(Q), ctypes.byref(it), ctypes.byref(ct)), lib)
    return Q, it.value, ct.value


def tecplot_write(path: str, ctime: float, pm: PlotMesh, plotq: np.ndarray, plotav=None) -> None:
    """tecpost_parallel's file from host plot-node values (9,plotnodes) and (2,plotnodes)."""
    lib = _lib()
    pq = np.asfortranarray(plotq, dtype=np.float64)
    pa = None if plotav is None else np.asfortranarray(plotav, dtype=np.float64)
    _check(lib.sddc_tecplot_write(str(path).encode(), float(ctime), pm.plotnodes, pm.plotcells, ptr(pm.plotx),
                                  ptr(pq), None if pa is None else ptr(pa), ptr(pm.connec, _I)), lib)
