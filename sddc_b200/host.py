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


def build_tables(mesh, N: int) -> Tables:
    lib = _lib()
    iv = np.asfortranarray(mesh.ivcell.astype(np.int32))
    xv = np.ascontiguousarray(mesh.xv, dtype=np.float64)
    yv = np.ascontiguousarray(mesh.yv, dtype=np.float64)
    bv = np.asfortranarray(mesh.bnd_v.astype(np.int32).reshape(-1, 2))
    bt = np.ascontiguousarray(mesh.bnd_type.astype(np.int32))
    h = ctypes.c_void_p()
    _check(lib.sddc_mesh_build(ctypes.byref(h), mesh.ncell, mesh.nvert, ptr(iv, _I), ptr(xv), ptr(yv),
                               int(bt.shape[0]), ptr(bv, _I), ptr(bt, _I), float(mesh.dxcycl),
                               float(mesh.dycycl)), lib)
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
        _check(lib.sddc_mesh_metrics(h, N, ptr(S1), ptr(S2), ptr(Jac), ptr(xx)), lib)
    finally:
        lib.sddc_mesh_destroy(h)
    Xs, Xf, L, M = sd_operators(N)
    return Tables(N=N, ncell=nc, Lmat=L, Mmat=M, Xs=Xs, Xf=Xf, S1=S1, S2=S2, Jac=Jac, xxsolu=xx, IF2C=IF2C,
                  IF2V=IF2V, ibfinter=lists["inter"], ibfinl=lists["inl"], ibfout=lists["out"],
                  ibfwal=lists["wal"], ibfsymp=lists["symp"], ibfree=lists["free"], cyc2fpair=cyc,
                  ivcell=ivc, counts=counts, dxcycl=float(mesh.dxcycl), dycycl=float(mesh.dycycl))
