"""ctypes binding of the CPU oracle (oracle/libsddc_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline / reference legs of bench.py; never by the product package.
Parity of this oracle against the reference itself is unpinned (the
reference has no golden vectors and no Fortran compiler exists here); it is
pinned by the known-answer tests in tests/test_oracle_kat.py.

``Oracle(..., tangent=True)`` loads the complex-step build of the same source
(libsddc_oracle_cs.so): its state arrays are complex128, and a state
Q + 1j*h*V evaluated with h ~ 1e-30 carries the FP64 tangent dR/dQ . V in
its imaginary part divided by h.

``Oracle(..., count=True)`` loads the operation-count build
(libsddc_oracle_count.so, the same source as C++ with a counting double):
``op_counts()`` returns the +/-, *, / and square roots applied to
state-dependent quantities since the last reset.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsddc_oracle.so")
LIB_CS = os.path.join(HERE, "libsddc_oracle_cs.so")
LIB_COUNT = os.path.join(HERE, "libsddc_oracle_count.so")

_I = ctypes.c_int
_L = ctypes.c_long
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)


class Params(ctypes.Structure):
    _fields_ = [("N", _I), ("ncell", _I), ("ncellglob", _I), ("vismode", _I), ("artiv", _I),
                ("skip_ideal_viscous", _I), ("mu", _D), ("eta0", _D), ("dxcycl", _D), ("dycycl", _D),
                ("rinf", _D), ("pinf", _D), ("uinf", _D), ("vinf", _D), ("bxinf", _D), ("byinf", _D)]


_libs = {}


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def _load(path, tangent, count=False):
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    L.orc_create.restype = ctypes.c_void_p
    L.orc_create.argtypes = [ctypes.POINTER(Params)]
    L.orc_destroy.argtypes = [ctypes.c_void_p]
    L.orc_set_threads.argtypes = [_I]
    L.orc_set_tables.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD, _PI, _I] + [_PI, _I] * 7
    L.orc_set_state.argtypes = [ctypes.c_void_p, _PD, _D, _D, _D]
    L.orc_get_state.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD]
    L.orc_set_freestream.argtypes = [ctypes.c_void_p, _PD]
    L.orc_get_maxima.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD]
    L.orc_get_fluxes.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD]
    L.orc_compresid.argtypes = [ctypes.c_void_p]
    L.orc_rk_s5p3.argtypes = [ctypes.c_void_p, _D, _I]
    L.orc_five_stage_rk.argtypes = [ctypes.c_void_p, _D, _I]
    L.orc_monitor.argtypes = [ctypes.c_void_p, _PD, _PD]
    L.orc_wall_force.argtypes = [ctypes.c_void_p, _PD, _PD, _PD]
    L.orc_setsandpoints.argtypes = [_I, _PD, _PD]
    L.orc_compute_LM.argtypes = [_I, _PD, _PD, _PD, _PD]
    L.orc_calcjacob_bilinear.argtypes = [_I, _I, _PI, _PD, _PD, _PD, _PD, _PD]
    L.orc_set_proc_faces.argtypes = [ctypes.c_void_p, _I, _PI]
    L.orc_proc_pack.argtypes = [ctypes.c_void_p, _PD]
    L.orc_proc_unpack.argtypes = [ctypes.c_void_p, _PD]
    L.orc_compresid_local.argtypes = [ctypes.c_void_p]
    L.orc_get_local_maxima.argtypes = [ctypes.c_void_p, _PD, _PD]
    L.orc_set_global_maxima.argtypes = [ctypes.c_void_p, _D, _D]
    L.orc_compresid_finish.argtypes = [ctypes.c_void_p]
    L.orc_rk_s5p3_begin_stage.argtypes = [ctypes.c_void_p, _I]
    L.orc_rk_s5p3_end_stage.argtypes = [ctypes.c_void_p, _I, _D]
    if count:  # the operation-count build: the residual path only
        L.orc_count_read.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), _I]
        return L
    if not tangent:  # complex scalars by value have no ctypes type; output routines: plain build
        L.orc_plot_setup.argtypes = [_I, _I, _PI, _PD, _PD, _PD, _PI, _I, _I, _PI, _PI, _PD, _PI, _PI, _PI]
        L.orc_calcjacob_8node.argtypes = [_I, _I, _PD, _PD, _PD, _PD]
        L.orc_plot_eval.argtypes = [_I, _I, _PD, _PD, _I, _I, _PI, _PI, _PD, _PD]
        L.orc_point_iflux.argtypes = [_PD, _D, _PD, _PD, _PD]
        L.orc_point_rusanov.argtypes = [_PD, _PD, _PD, _PD, _PD, _I, _I, _D, _PD, _PD, _PD]
        L.orc_rk_s5p3_combine.argtypes = [_I, _L, _D, _PD, _PD, _PD, _PD]
    return L


def lib(tangent: bool = False, count: bool = False):
    key = "count" if count else tangent
    if key not in _libs:
        _libs[key] = _load(LIB_COUNT if count else (LIB_CS if tangent else LIB), tangent, count)
    return _libs[key]


def _p(a, t=_PD):
    return None if a is None else a.ctypes.data_as(t)


def set_threads(n: int) -> None:
    lib()
    for L in _libs.values():
        L.orc_set_threads(int(n))


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
    """The reference's single-rank residual path on the CPU, FP64 (or its
    complex-step tangent with ``tangent=True``, or the operation-count build
    with ``count=True``)."""

    def __init__(self, tables, physics, skip_ideal_viscous: bool = False, ncellglob: int | None = None,
                 tangent: bool = False, count: bool = False):
        if tangent and count:
            raise ValueError("the tangent and operation-count builds are separate")
        self.N = tables.N
        self.ncell = tables.ncell
        self.tangent = tangent
        self.count = count
        self._L = lib(tangent, count)
        self.dtype = np.complex128 if tangent else np.float64
        p = Params(N=tables.N, ncell=tables.ncell, ncellglob=ncellglob or tables.ncell, vismode=physics.vismode,
                   artiv=physics.artiv, skip_ideal_viscous=int(skip_ideal_viscous), mu=physics.mu,
                   eta0=physics.eta0, dxcycl=physics.dxcycl, dycycl=physics.dycycl, rinf=physics.rinf,
                   pinf=physics.pinf, uinf=physics.uinf, vinf=physics.vinf, bxinf=physics.bxinf,
                   byinf=physics.byinf)
        self._h = self._L.orc_create(ctypes.byref(p))
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
        self._L.orc_set_tables(self._h, _p(np.asfortranarray(t.Lmat)), _p(np.asfortranarray(t.Mmat)),
                               _p(np.asfortranarray(t.S1)), _p(np.asfortranarray(t.S2)),
                               _p(np.asfortranarray(t.Jac)), _p(if2c, _PI), t.nface, *args)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.orc_destroy(h)
            self._h = None

    def _arr(self, shape):
        return np.zeros(shape, dtype=self.dtype, order="F")

    def set_state(self, Q, ctime=0.0, eigvmax=0.0, umax=0.0):
        Q = np.asfortranarray(Q, dtype=self.dtype)
        self._L.orc_set_state(self._h, _p(Q), ctime, eigvmax, umax)

    def set_freestream(self, fs):
        """Boundary free stream (rinf, pinf, uinf, vinf, bxinf, byinf)."""
        fs = np.ascontiguousarray(fs, dtype=self.dtype)
        assert fs.shape == (6,)
        self._L.orc_set_freestream(self._h, _p(fs))

    def op_counts(self, reset: bool = True) -> dict:
        """Operations on state-dependent quantities since the last reset
        (operation-count build only): add (+ and -), mul, div, sqrt."""
        if not self.count:
            raise ValueError("op_counts needs Oracle(..., count=True)")
        out = (ctypes.c_ulonglong * 4)()
        self._L.orc_count_read(out, int(reset))
        return {"add": out[0], "mul": out[1], "div": out[2], "sqrt": out[3]}

    def compresid(self):
        self._L.orc_compresid(self._h)

    def rk_s5p3(self, dt, nsteps=1):
        self._L.orc_rk_s5p3(self._h, dt, nsteps)

    def five_stage_rk(self, dt, nsteps=1):
        self._L.orc_five_stage_rk(self._h, dt, nsteps)

    def state(self):
        N, nc = self.N, self.ncell
        Q = self._arr((9, N, N, nc))
        R = self._arr((9, N, N, nc))
        G = self._arr((9, 2, N, N, nc))
        mu = np.zeros((2, nc), order="F")
        sm = np.zeros((2, nc), order="F")
        self._L.orc_get_state(self._h, _p(Q), _p(R), _p(G), _p(mu), _p(sm))
        return dict(Q=Q, resid=R, nablaQs=G, muAV=mu, sm_ind=sm)

    def fluxes(self):
        N, nc = self.N, self.ncell
        out = [self._arr((9, N + 1, N, nc)), self._arr((9, N, N + 1, nc)),
               self._arr((9, N + 1, N, nc)), self._arr((9, N, N + 1, nc))]
        self._L.orc_get_fluxes(self._h, *[_p(a) for a in out])
        return dict(F1=out[0], G2=out[1], Fv1=out[2], Gv2=out[3])

    def maxima(self):
        v = [_D() for _ in range(5)]
        self._L.orc_get_maxima(self._h, *[ctypes.byref(x) for x in v])
        return dict(eigvmax=v[0].value, umax=v[1].value, c_h=v[2].value, epsilon0=v[3].value,
                    ctime=v[4].value)

    def monitor(self):
        a, b = _D(), _D()
        self._L.orc_monitor(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    # -- decomposed runs: one rank of a partitioned case ---------------------
    def set_proc_faces(self, ibfproc):
        """The processor faces (local face ids, 1-based, in slot order)."""
        self._ibfproc = np.ascontiguousarray(ibfproc, dtype=np.int32)
        rc = self._L.orc_set_proc_faces(self._h, len(self._ibfproc), _p(self._ibfproc, _PI))
        if rc:
            raise ValueError("orc_set_proc_faces rejected the list")

    def proc_pack(self):
        """The send buffer (nproc, N, 9): own traces, nfp ascending."""
        buf = np.zeros((len(self._ibfproc), self.N, 9), dtype=self.dtype)
        self._L.orc_proc_pack(self._h, _p(buf))
        return buf

    def proc_unpack(self, rbuf):
        rbuf = np.ascontiguousarray(rbuf, dtype=self.dtype)
        assert rbuf.shape == (len(self._ibfproc), self.N, 9)
        self._L.orc_proc_unpack(self._h, _p(rbuf))

    def compresid_local(self):
        self._L.orc_compresid_local(self._h)

    def local_maxima(self):
        e, u = _D(), _D()
        self._L.orc_get_local_maxima(self._h, ctypes.byref(e), ctypes.byref(u))
        return e.value, u.value

    def set_global_maxima(self, eigvmax, umax):
        self._L.orc_set_global_maxima(self._h, float(eigvmax), float(umax))

    def compresid_finish(self):
        self._L.orc_compresid_finish(self._h)

    def rk_begin_stage(self, stage):
        self._L.orc_rk_s5p3_begin_stage(self._h, int(stage))

    def rk_end_stage(self, stage, dt):
        self._L.orc_rk_s5p3_end_stage(self._h, int(stage), float(dt))

    def wall_force(self, w):
        """(Fx, Fy) on the wall faces at the current state; w = quadrature
        weights of the N solution points on [0, 1]."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert w.shape == (self.N,)
        fx, fy = np.zeros(1, dtype=self.dtype), np.zeros(1, dtype=self.dtype)
        self._L.orc_wall_force(self._h, _p(w), _p(fx), _p(fy))
        return fx[0], fy[0]


def sp_weights(Xs):
    """Quadrature weights of the solution points on [0, 1] (integrals of the
    Lagrange basis): the moment equations sum_i w_i Xs_i^k = 1/(k+1)."""
    Xs = np.asarray(Xs, dtype=np.float64)
    N = Xs.size
    A = np.vander(Xs, N, increasing=True).T
    b = 1.0 / np.arange(1, N + 1)
    return np.linalg.solve(A, b)


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


# ---------------------------------------------------------------- output
# tecplotter2dsetup / tecplotter2d (sddc_oracle_output.c) and a numpy
# restatement of the file formats of tecpost_parallel (tecplotter.f90:99-415)
# and WRITE_ALL_DATA_PARALLEL (write_data.f90:1-83), independent of the
# product's writers.

def metrics8(N: int, xxf_cell: np.ndarray):
    """calcjacob with 8-node cells (CURVE_WALL = 1): (S1, S2, Jac)."""
    nc = xxf_cell.shape[2]
    xx = np.asfortranarray(xxf_cell, dtype=np.float64)
    S1 = np.zeros((2, 2, N + 1, N, nc), order="F")
    S2 = np.zeros((2, 2, N, N + 1, nc), order="F")
    J = np.zeros((N, N, nc), order="F")
    lib().orc_calcjacob_8node(N, nc, _p(xx), _p(S1), _p(S2), _p(J))
    return S1, S2, J


def plot_setup(ivcell, xv, yv, if2c, nre, xxf_cell=None):
    """(plotnodes, plotcells, plotX (2,.), gnumnode, gnode_factor, connec (4,.))."""
    nc = ivcell.shape[0]
    cap = (nre + 1) ** 2 * nc
    iv = np.asfortranarray(ivcell, dtype=np.int32)
    f2c = np.asfortranarray(if2c, dtype=np.int32)
    px = np.zeros((2, cap), order="F")
    gn = np.zeros((nre + 1, nre + 1, nc), np.int32, order="F")
    gf = np.zeros(cap, np.int32)
    cn = np.zeros((4, nre * nre * nc), np.int32, order="F")
    nn, ncl = ctypes.c_int(), ctypes.c_int()
    xx = None if xxf_cell is None else np.asfortranarray(xxf_cell, dtype=np.float64)
    rc = lib().orc_plot_setup(nc, len(xv), _p(iv, _PI), _p(np.ascontiguousarray(xv, dtype=np.float64)),
                              _p(np.ascontiguousarray(yv, dtype=np.float64)), _p(xx), _p(f2c, _PI),
                              f2c.shape[0], nre,
                              ctypes.byref(nn), ctypes.byref(ncl), _p(px), _p(gn, _PI), _p(gf, _PI), _p(cn, _PI))
    if rc != 0:
        raise RuntimeError(f"orc_plot_setup failed ({rc})")
    n = nn.value
    return n, ncl.value, np.asfortranarray(px[:, :n]), gn, gf[:n].copy(), cn


def plot_eval(N, Q, muAV, nre, plotnodes, gnumnode, gnode_factor):
    """tecplotter2d: (plotQ (9,plotnodes), plotAV (2,plotnodes))."""
    nc = Q.shape[3]
    q = np.asfortranarray(Q, dtype=np.float64)
    mu = None if muAV is None else np.asfortranarray(muAV, dtype=np.float64)
    pq = np.zeros((9, plotnodes), order="F")
    pa = np.zeros((2, plotnodes), order="F")
    lib().orc_plot_eval(N, nc, _p(q), _p(mu), nre, plotnodes, _p(np.asfortranarray(gnumnode, dtype=np.int32), _PI),
                        _p(np.ascontiguousarray(gnode_factor, dtype=np.int32), _PI), _p(pq), _p(pa))
    return pq, pa


def _fortran_fixed(x, d):
    """Digits of Fw.d for 0 <= x < 1 from the exact binary value, ties away from zero."""
    from fractions import Fraction
    t = Fraction(x) * 10 ** d
    fl = t.numerator // t.denominator
    r = t - fl
    return fl + (1 if r >= Fraction(1, 2) else 0)


def restart_name(it):
    return f"restart.{it:08d}.dat"


def tecplot_name(ctime):
    ip = int(ctime)
    d = _fortran_fixed(ctime - ip, 3)
    return f"TEC{ip:07d}.{d % 1000:03d}.plt"


def restart_bytes(it, ctime, Q, icg=None):
    nv, n, _, nc = Q.shape
    rec = np.dtype([("icg", "<i4"), ("q", "<f8", (nv * n * n,))])
    body = np.zeros(nc, dtype=rec)
    body["icg"] = np.arange(1, nc + 1) if icg is None else icg
    body["q"] = np.asfortranarray(Q).reshape(nv * n * n, nc, order="F").T
    return np.int32(it).tobytes() + np.float64(ctime).tobytes() + body.tobytes()


def _tec_string(s):
    return np.array([ord(c) for c in s] + [0], dtype="<i4").tobytes()


def tecplot_bytes(ctime, plotx, plotq, plotav, connec):
    names = ["X", "Y", "RHO", "U", "V", "W", "P", "Bx", "By", "Bz", "Az", "muAV", "etaAV"]
    nn, ncl = plotx.shape[1], connec.shape[1]
    av = np.zeros((2, nn)) if plotav is None else plotav
    vals = [plotx[0], plotx[1]] + [plotq[k] for k in range(9)] + [av[0], av[1]]
    out = [b"#!TDV111", np.array([1, 0], "<i4").tobytes(), _tec_string("step data"),
           np.int32(len(names)).tobytes()]
    out += [_tec_string(n) for n in names]
    out += [np.float32(299.0).tobytes(), _tec_string("ZONE 001"), np.array([-1, 0], "<i4").tobytes(),
            np.float64(ctime).tobytes(), np.array([-1, 3, 0, 0, 0, 0, nn, ncl, 0, 0, 0, 0], "<i4").tobytes(),
            np.float32(357.0).tobytes(), np.float32(299.0).tobytes(),
            np.array([1] * len(names) + [0, 0, -1], "<i4").tobytes()]
    mm = np.array([[v.min(), v.max()] for v in vals], dtype="<f8")
    out.append(mm.tobytes())
    out += [np.asarray(v, dtype="<f4").tobytes() for v in vals]
    out.append((np.asfortranarray(connec).T.astype("<i4") - 1).tobytes())
    return b"".join(out)
