"""ctypes binding of the CPU oracle (oracle/libsddc_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline / reference legs of bench.py; never by the product package.
Parity of this oracle against the reference itself is unpinned (the
reference has no golden vectors and no Fortran compiler exists here); it is
pinned by the known-answer tests in tests/test_oracle_kat.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsddc_oracle.so")

_I = ctypes.c_int
_L = ctypes.c_long
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)


class Params(ctypes.Structure):
    _fields_ = [("N", _I), ("ncell", _I), ("ncellglob", _I), ("vismode", _I), ("artiv", _I),
                ("skip_ideal_viscous", _I), ("mu", _D), ("eta0", _D), ("dxcycl", _D), ("dycycl", _D),
                ("rinf", _D), ("pinf", _D), ("uinf", _D), ("vinf", _D), ("bxinf", _D), ("byinf", _D)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(Params)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [_I]
        L.orc_set_tables.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD, _PI, _I] + [_PI, _I] * 7
        L.orc_set_state.argtypes = [ctypes.c_void_p, _PD, _D, _D, _D]
        L.orc_get_state.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD]
        L.orc_get_maxima.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD]
        L.orc_get_fluxes.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD]
        L.orc_compresid.argtypes = [ctypes.c_void_p]
        L.orc_rk_s5p3.argtypes = [ctypes.c_void_p, _D, _I]
        L.orc_five_stage_rk.argtypes = [ctypes.c_void_p, _D, _I]
        L.orc_monitor.argtypes = [ctypes.c_void_p, _PD, _PD]
        L.orc_setsandpoints.argtypes = [_I, _PD, _PD]
        L.orc_compute_LM.argtypes = [_I, _PD, _PD, _PD, _PD]
        L.orc_calcjacob_bilinear.argtypes = [_I, _I, _PI, _PD, _PD, _PD, _PD, _PD]
        L.orc_point_iflux.argtypes = [_PD, _D, _PD, _PD, _PD]
        L.orc_point_rusanov.argtypes = [_PD, _PD, _PD, _PD, _PD, _I, _I, _D, _PD, _PD, _PD]
        L.orc_rk_s5p3_combine.argtypes = [_I, _L, _D, _PD, _PD, _PD, _PD]
        _lib = L
    return _lib


def _p(a, t=_PD):
    return None if a is None else a.ctypes.data_as(t)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def operators(N: int):
    L = lib()
    Xs, Xf = np.zeros(N), np.zeros(N + 1)
    L.orc_setsandpoints(N, _p(Xs), _p(Xf))
    Lm = np.zeros((N + 1, N), order="F")
    Mm = np.zeros((N + 1, N), order="F")
    L.orc_compute_LM(N, _p(Xs), _p(Xf), _p(Lm), _p(Mm))
    return Xs, Xf, Lm, Mm


def metrics(N: int, ivcell: np.ndarray, xv: np.ndarray, yv: np.ndarray):
    nc = ivcell.shape[0]
    iv = np.asfortranarray(ivcell.astype(np.int32))
    S1 = np.zeros((2, 2, N + 1, N, nc), order="F")
    S2 = np.zeros((2, 2, N, N + 1, nc), order="F")
    J = np.zeros((N, N, nc), order="F")
    lib().orc_calcjacob_bilinear(N, nc, _p(iv, _PI), _p(np.ascontiguousarray(xv)), _p(np.ascontiguousarray(yv)),
                                 _p(S1), _p(S2), _p(J))
    return S1, S2, J


class Oracle:
    """The reference's single-rank residual path on the CPU, FP64."""

    def __init__(self, tables, physics, skip_ideal_viscous: bool = False, ncellglob: int | None = None):
        self.N = tables.N
        self.ncell = tables.ncell
        p = Params(N=tables.N, ncell=tables.ncell, ncellglob=ncellglob or tables.ncell, vismode=physics.vismode,
                   artiv=physics.artiv, skip_ideal_viscous=int(skip_ideal_viscous), mu=physics.mu,
                   eta0=physics.eta0, dxcycl=physics.dxcycl, dycycl=physics.dycycl, rinf=physics.rinf,
                   pinf=physics.pinf, uinf=physics.uinf, vinf=physics.vinf, bxinf=physics.bxinf,
                   byinf=physics.byinf)
        self._h = lib().orc_create(ctypes.byref(p))
        if not self._h:
            raise ValueError("orc_create rejected the parameters")
        t = tables
        ints = [(np.asfortranarray(a, dtype=np.int32), n) for a, n in (
            (t.ibfinter, len(t.ibfinter)), (t.ibfinl, len(t.ibfinl)), (t.ibfout, len(t.ibfout)),
            (t.ibfwal, len(t.ibfwal)), (t.ibfsymp, len(t.ibfsymp)), (t.ibfree, len(t.ibfree)),
            (t.cyc2fpair, int(t.cyc2fpair.shape[0])))]
        self._keep = ints
        args = []
        for a, n in ints:
            args += [_p(a, _PI), n]
        if2c = np.asfortranarray(t.IF2C, dtype=np.int32)
        self._keep.append(if2c)
        lib().orc_set_tables(self._h, _p(np.asfortranarray(t.Lmat)), _p(np.asfortranarray(t.Mmat)),
                             _p(np.asfortranarray(t.S1)), _p(np.asfortranarray(t.S2)),
                             _p(np.asfortranarray(t.Jac)), _p(if2c, _PI), t.nface, *args)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def set_state(self, Q, ctime=0.0, eigvmax=0.0, umax=0.0):
        Q = np.asfortranarray(Q, dtype=np.float64)
        lib().orc_set_state(self._h, _p(Q), ctime, eigvmax, umax)

    def compresid(self):
        lib().orc_compresid(self._h)

    def rk_s5p3(self, dt, nsteps=1):
        lib().orc_rk_s5p3(self._h, dt, nsteps)

    def five_stage_rk(self, dt, nsteps=1):
        lib().orc_five_stage_rk(self._h, dt, nsteps)

    def state(self):
        N, nc = self.N, self.ncell
        Q = np.zeros((9, N, N, nc), order="F")
        R = np.zeros((9, N, N, nc), order="F")
        G = np.zeros((9, 2, N, N, nc), order="F")
        mu = np.zeros((2, nc), order="F")
        sm = np.zeros((2, nc), order="F")
        lib().orc_get_state(self._h, _p(Q), _p(R), _p(G), _p(mu), _p(sm))
        return dict(Q=Q, resid=R, nablaQs=G, muAV=mu, sm_ind=sm)

    def fluxes(self):
        N, nc = self.N, self.ncell
        out = [np.zeros((9, N + 1, N, nc), order="F"), np.zeros((9, N, N + 1, nc), order="F"),
               np.zeros((9, N + 1, N, nc), order="F"), np.zeros((9, N, N + 1, nc), order="F")]
        lib().orc_get_fluxes(self._h, *[_p(a) for a in out])
        return dict(F1=out[0], G2=out[1], Fv1=out[2], Gv2=out[3])

    def maxima(self):
        v = [_D() for _ in range(5)]
        lib().orc_get_maxima(self._h, *[ctypes.byref(x) for x in v])
        return dict(eigvmax=v[0].value, umax=v[1].value, c_h=v[2].value, epsilon0=v[3].value,
                    ctime=v[4].value)

    def monitor(self):
        a, b = _D(), _D()
        lib().orc_monitor(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value


def point_iflux(q, c_h=0.0):
    q = np.ascontiguousarray(q, dtype=np.float64)
    F, G = np.zeros(9), np.zeros(9)
    um = _D(0.0)
    lib().orc_point_iflux(_p(q), c_h, ctypes.byref(um), _p(F), _p(G))
    return F, G, um.value


def point_rusanov(ql, qr, normf, sign_l=1, sign_r=1, c_h=0.0):
    ql = np.ascontiguousarray(ql, dtype=np.float64)
    qr = np.ascontiguousarray(qr, dtype=np.float64)
    nf = np.ascontiguousarray(normf, dtype=np.float64)
    Fl, Fr = np.zeros(9), np.zeros(9)
    ev, em, um = _D(), _D(0.0), _D(0.0)
    lib().orc_point_rusanov(_p(ql), _p(qr), _p(Fl), _p(Fr), _p(nf), sign_l, sign_r, c_h, ctypes.byref(ev),
                            ctypes.byref(em), ctypes.byref(um))
    return Fl, Fr, ev.value, um.value


def rk_s5p3_combine(stage, dt, q, qk0, qka, r):
    q = np.ascontiguousarray(q, dtype=np.float64)
    lib().orc_rk_s5p3_combine(stage, q.size, dt, _p(q), _p(np.ascontiguousarray(qk0, dtype=np.float64)),
                              _p(np.ascontiguousarray(qka, dtype=np.float64)),
                              _p(np.ascontiguousarray(r, dtype=np.float64)))
    return q
