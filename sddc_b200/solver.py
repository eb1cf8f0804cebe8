"""The drop-in, driven from Python through its C ABI (include/sddc.h).

``Solver`` mirrors what the reference's Fortran host does around the hot
path: it passes the set-up tables once (``sddc_set_tables``), the state
(``sddc_set_state``, the restart route of initsetup.f90:154-162), then calls
``compresid`` or ``rk_s5p3`` (RK_S5P3, iterations.f90:158-213) and reads
results back.  ``iterations`` replays the reference's time loop with its
residual monitor (iterations.f90:19-83).

There is no CPU path: a missing or unloadable ``libsddc_b200.so`` raises.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _native
from ._native import ptr

_I = ctypes.c_int
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)

FP64_EXACT, FP64, MIXED = 0, 1, 2
PRECISIONS = {"fp64_exact": FP64_EXACT, "fp64": FP64, "mixed": MIXED}

OK, EINVAL, ECUDA, ESTATE, ENUMERIC, ENOMEM, EIO = 0, -1, -2, -3, -4, -5, -6

EXPORTED = ("sddc_create", "sddc_destroy", "sddc_last_error", "sddc_set_tables", "sddc_set_state",
            "sddc_compresid", "sddc_rk_step", "sddc_get_state", "sddc_monitor", "sddc_get_maxima",
            "sddc_state_device_ptr", "sddc_get_stream", "sddc_set_cases", "sddc_rk_step_cases",
            "sddc_get_case_maxima", "sddc_vjp_resid", "sddc_adjoint_run", "sddc_set_plot", "sddc_plot_nodes",
            "sddc_write_tecplot", "sddc_write_restart", "sddc_output_wait", "sddc_set_proc_faces",
            "sddc_set_exchange", "sddc_set_persistent")


class Params(ctypes.Structure):
    _fields_ = [("N", _I), ("ncell", _I), ("ncellglob", _I), ("vismode", _I), ("artiv", _I), ("k_stage", _I),
                ("precision", _I), ("cells_per_cta", _I), ("mu", _D), ("eta0", _D), ("dxcycl", _D),
                ("dycycl", _D), ("rinf", _D), ("pinf", _D), ("uinf", _D), ("vinf", _D), ("bxinf", _D),
                ("byinf", _D)]


class CaseRecord(ctypes.Structure):
    """sddc_case: one case of a batch."""
    _fields_ = [("first_cell", _I), ("ncell", _I), ("dt", _D), ("rinf", _D), ("pinf", _D), ("uinf", _D),
                ("vinf", _D), ("bxinf", _D), ("byinf", _D)]


class AdjointOpts(ctypes.Structure):
    """sddc_adjoint_opts."""
    _fields_ = [("dt", _D), ("nsteps", _I), ("n1", _I), ("n2", _I), ("w_drag", _D), ("w_lift", _D),
                ("diameter", _D), ("checkpoint_every", _I)]


class AdjointStats(ctypes.Structure):
    """sddc_adjoint_stats."""
    _fields_ = [("forward_ms", _D), ("reverse_ms", _D), ("device_bytes", _D), ("owner_stages", _I),
                ("tie_stages", _I)]


# int (*sddc_exchange_fn)(void *user)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


class SddcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sddc error {code}: {msg}")
        self.code = code


class NumericalFault(SddcError):
    """The device saw a non-positive density or a non-finite wave speed."""


def lib():
    L = _native.load(_native.GPU_LIB)
    if not getattr(L, "_sddc_typed", False):
        L.sddc_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Params)]
        L.sddc_destroy.argtypes = [ctypes.c_void_p]
        L.sddc_destroy.restype = None
        L.sddc_last_error.argtypes = [ctypes.c_void_p]
        L.sddc_last_error.restype = ctypes.c_char_p
        L.sddc_set_tables.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD, _PI, _I] + [_PI, _I] * 7
        L.sddc_set_state.argtypes = [ctypes.c_void_p, _PD, _D, _D, _D]
        L.sddc_compresid.argtypes = [ctypes.c_void_p]
        L.sddc_rk_step.argtypes = [ctypes.c_void_p, _D, _I]
        L.sddc_get_state.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD, _PD]
        L.sddc_monitor.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD]
        L.sddc_get_maxima.argtypes = [ctypes.c_void_p, _PD, _PD, _PD, _PD]
        L.sddc_state_device_ptr.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.sddc_get_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.sddc_set_cases.argtypes = [ctypes.c_void_p, _I, ctypes.POINTER(CaseRecord)]
        L.sddc_rk_step_cases.argtypes = [ctypes.c_void_p, _I]
        L.sddc_get_case_maxima.argtypes = [ctypes.c_void_p, _I, _PD, _PD]
        L.sddc_vjp_resid.argtypes = [ctypes.c_void_p, _PD, _PD, _PD]
        L.sddc_adjoint_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(AdjointOpts), _PD, _PD, _PD,
                                       ctypes.POINTER(AdjointStats)]
        L.sddc_set_plot.argtypes = [ctypes.c_void_p, _I, _I, _I, _PD, _PI, _PI, _PI]
        L.sddc_plot_nodes.argtypes = [ctypes.c_void_p, _PD, _PD]
        L.sddc_write_tecplot.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.sddc_write_restart.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _I, _PI]
        L.sddc_output_wait.argtypes = [ctypes.c_void_p]
        L.sddc_set_proc_faces.argtypes = [ctypes.c_void_p, _I, _PI]
        L.sddc_set_persistent.argtypes = [ctypes.c_void_p, _I]
        L.sddc_set_exchange.argtypes = [ctypes.c_void_p, EXCHANGE_FN, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        L._sddc_typed = True
    return L


class Solver:
    """One case on the current GPU."""

    def __init__(self, tables, physics, precision="fp64", k_stage: int = 3, cells_per_cta: int = 0,
                 ncellglob: int | None = None, proc_faces=None):
        """proc_faces: the processor faces of one partition of a decomposed
        run (local face ids, 1-based, in exchange-slot order; see
        partition.Part); the exchange follows with set_exchange."""
        self.N = tables.N
        self.ncell = tables.ncell
        self.tables = tables
        self.physics = physics
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.k_stage = k_stage
        p = Params(N=tables.N, ncell=tables.ncell, ncellglob=ncellglob or tables.ncell, vismode=physics.vismode,
                   artiv=physics.artiv, k_stage=k_stage, precision=self.precision, cells_per_cta=cells_per_cta,
                   mu=physics.mu, eta0=physics.eta0, dxcycl=physics.dxcycl, dycycl=physics.dycycl,
                   rinf=physics.rinf, pinf=physics.pinf, uinf=physics.uinf, vinf=physics.vinf,
                   bxinf=physics.bxinf, byinf=physics.byinf)
        self._L = lib()
        self._h = ctypes.c_void_p()
        rc = self._L.sddc_create(ctypes.byref(self._h), ctypes.byref(p))
        if rc != OK:
            msg = self._L.sddc_last_error(self._h).decode() if self._h else "sddc_create failed"
            self.close()
            raise SddcError(rc, msg)
        t = tables
        keep = []
        if proc_faces is not None:
            pf = np.ascontiguousarray(proc_faces, dtype=np.int32)
            keep.append(pf)
            self._check(self._L.sddc_set_proc_faces(self._h, int(pf.shape[0]), ptr(pf, _I)))

        def ia(a):
            a = np.asfortranarray(a, dtype=np.int32)
            keep.append(a)
            return ptr(a, _I)

        def da(a):
            a = np.asfortranarray(a, dtype=np.float64)
            keep.append(a)
            return ptr(a)

        self._check(self._L.sddc_set_tables(
            self._h, da(t.Lmat), da(t.Mmat), da(t.S1), da(t.S2), da(t.Jac), ia(t.IF2C), t.nface,
            ia(t.ibfinter), len(t.ibfinter), ia(t.ibfinl), len(t.ibfinl), ia(t.ibfout), len(t.ibfout),
            ia(t.ibfwal), len(t.ibfwal), ia(t.ibfsymp), len(t.ibfsymp), ia(t.ibfree), len(t.ibfree),
            ia(t.cyc2fpair), int(t.cyc2fpair.shape[0])))

    # -- plumbing ----------------------------------------------------------
    def _check(self, rc):
        if rc == OK:
            return
        msg = self._L.sddc_last_error(self._h).decode()
        if rc == ENUMERIC:
            raise NumericalFault(rc, msg)
        raise SddcError(rc, msg)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.sddc_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the reference-facing calls -----------------------------------------
    def set_state(self, Q, ctime=0.0, eigvmax=0.0, umax=0.0):
        Q = np.asfortranarray(Q, dtype=np.float64)
        assert Q.shape == (9, self.N, self.N, self.ncell)
        self._check(self._L.sddc_set_state(self._h, ptr(Q), ctime, eigvmax, umax))

    def compresid(self):
        self._check(self._L.sddc_compresid(self._h))

    def rk_s5p3(self, dt, nsteps=1):
        """nsteps time steps with the context's scheme (k_stage 3 or 5)."""
        self._check(self._L.sddc_rk_step(self._h, float(dt), int(nsteps)))

    step = rk_s5p3

    def state(self, resid=False, nablaQs=False, muAV=False, sm_ind=False, out=None):
        N, nc = self.N, self.ncell
        Q = out if out is not None else np.zeros((9, N, N, nc), order="F")
        R = np.zeros((9, N, N, nc), order="F") if resid else None
        G = np.zeros((9, 2, N, N, nc), order="F") if nablaQs else None
        M = np.zeros((2, nc), order="F") if muAV else None
        S = np.zeros((2, nc), order="F") if sm_ind else None
        self._check(self._L.sddc_get_state(self._h, ptr(Q), ptr(R), ptr(G), ptr(M), ptr(S)))
        d = dict(Q=Q)
        for k, v in (("resid", R), ("nablaQs", G), ("muAV", M), ("sm_ind", S)):
            if v is not None:
                d[k] = v
        return d

    def monitor(self):
        v = [_D() for _ in range(4)]
        self._check(self._L.sddc_monitor(self._h, *[ctypes.byref(x) for x in v]))
        return dict(residsum=v[0].value, divbsum=v[1].value, mass=v[2].value, energy=v[3].value)

    def maxima(self):
        v = [_D() for _ in range(4)]
        self._check(self._L.sddc_get_maxima(self._h, *[ctypes.byref(x) for x in v]))
        return dict(eigvmax=v[0].value, umax=v[1].value, c_h=v[2].value, ctime=v[3].value)

    def device_state_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._L.sddc_state_device_ptr(self._h, ctypes.byref(p)))
        return p.value

    def stream_handle(self) -> int:
        """The cudaStream_t of the context (for CUDA events around its work)."""
        p = ctypes.c_void_p()
        self._check(self._L.sddc_get_stream(self._h, ctypes.byref(p)))
        return p.value

    # -- decomposed runs -----------------------------------------------------
    def set_exchange(self, fn, send_ptr: int, recv_ptr: int, maxima_ptr: int):
        """fn(user) -> int is called between stages, on the context's stream,
        after the library wrote this rank's processor-face traces to the
        device buffer at send_ptr and its running maxima to maxima_ptr; it
        exchanges the traces into recv_ptr and reduces the maxima (MAX) in
        place, and returns 0."""
        def tramp(user):
            try:
                return int(fn(user) or 0)
            except Exception:  # an exception cannot cross into C
                import traceback

                traceback.print_exc()
                return 1

        self._exchange_cb = EXCHANGE_FN(tramp)  # kept alive with the solver
        self._check(self._L.sddc_set_exchange(self._h, self._exchange_cb, None, ctypes.c_void_p(send_ptr),
                                              ctypes.c_void_p(recv_ptr), ctypes.c_void_p(maxima_ptr)))

    # -- batches of cases ---------------------------------------------------
    def set_cases(self, records):
        """records: sequence of dicts with first_cell, ncell, dt and the free
        stream (rinf, pinf, uinf, vinf, bxinf, byinf)."""
        arr = (CaseRecord * len(records))()
        for k, r in enumerate(records):
            for f, _ in CaseRecord._fields_:
                setattr(arr[k], f, r[f])
        self._check(self._L.sddc_set_cases(self._h, len(records), arr))
        self.ncase = len(records)

    def set_persistent(self, on=True):
        """Batch stages as persistent grid-stride launches (largest case
        first) instead of one CTA per tile."""
        self._check(self._L.sddc_set_persistent(self._h, int(bool(on))))

    def step_cases(self, nsteps=1):
        self._check(self._L.sddc_rk_step_cases(self._h, int(nsteps)))

    def case_maxima(self, icase):
        e, u = _D(), _D()
        self._check(self._L.sddc_get_case_maxima(self._h, int(icase), ctypes.byref(e), ctypes.byref(u)))
        return e.value, u.value

    # -- discrete adjoint -----------------------------------------------------
    def vjp_resid(self, Rbar):
        """(dR/dQ)^T Rbar at the current state (exact FP64 residual); returns
        (Qbar, parbar) with parbar = [Rbar . dR/dc_h, Rbar . dR/d(rinf, pinf,
        uinf, vinf, bxinf, byinf)]."""
        Rbar = np.asfortranarray(Rbar, dtype=np.float64)
        Qbar = np.zeros((9, self.N, self.N, self.ncell), order="F")
        par = np.zeros(7)
        self._check(self._L.sddc_vjp_resid(self._h, ptr(Rbar), ptr(Qbar), ptr(par)))
        return Qbar, par

    def adjoint_run(self, dt, nsteps, n1, n2, w_drag=1.0, w_lift=0.0, diameter=1.0, checkpoint_every=20,
                    gradient=True):
        """nsteps exact RK_S5P3 steps from the current state and the
        objective J = mean over the states after n1..n2 steps of
        w_drag*C_D + w_lift*C_L, with (gradient=True) dJ/dQ0 and dJ/d(free
        stream) by the discrete adjoint.  The context ends at the final
        state."""
        o = AdjointOpts(dt=dt, nsteps=int(nsteps), n1=int(n1), n2=int(n2), w_drag=w_drag, w_lift=w_lift,
                        diameter=diameter, checkpoint_every=int(checkpoint_every))
        obj = np.zeros(3)
        st = AdjointStats()
        Qbar = np.zeros((9, self.N, self.N, self.ncell), order="F") if gradient else None
        par = np.zeros(6) if gradient else None
        self._check(self._L.sddc_adjoint_run(self._h, ctypes.byref(o), ptr(obj), ptr(Qbar) if gradient else None,
                                             ptr(par) if gradient else None, ctypes.byref(st)))
        return dict(J=obj[0], cd=obj[1], cl=obj[2], Qbar0=Qbar, parbar=par,
                    stats={f: getattr(st, f) for f, _ in AdjointStats._fields_})

    # -- output from the device state ------------------------------------------
    def set_plot(self, pm):
        """The plot mesh of the Tecplot output (host.PlotMesh, tecplotter2dsetup)."""
        self._plot = pm
        self._check(self._L.sddc_set_plot(self._h, pm.nre, pm.plotnodes, pm.plotcells, ptr(pm.plotx),
                                          ptr(pm.gnumnode, _I), ptr(pm.gnode_factor, _I), ptr(pm.connec, _I)))

    def plot_nodes(self):
        """tecplotter2d on the device: (plotQ (9,plotnodes), plotAV (2,plotnodes))."""
        n = self._plot.plotnodes
        pq = np.zeros((9, n), order="F")
        pa = np.zeros((2, n), order="F")
        self._check(self._L.sddc_plot_nodes(self._h, ptr(pq), ptr(pa)))
        return pq, pa

    def write_tecplot(self, path=None):
        """Queues the Tecplot file of the current state (tecpost_parallel's format)."""
        self._check(self._L.sddc_write_tecplot(self._h, None if path is None else str(path).encode()))

    def write_restart(self, path=None, iter_=0, icg=None):
        """Queues the restart file of the current state (WRITE_ALL_DATA_PARALLEL's format)."""
        g = None if icg is None else np.ascontiguousarray(icg, dtype=np.int32)
        self._check(self._L.sddc_write_restart(self._h, None if path is None else str(path).encode(), int(iter_),
                                               ptr(g, _I)))

    def output_wait(self):
        """Blocks until every queued file is written; raises the first failure."""
        self._check(self._L.sddc_output_wait(self._h))

    # -- the reference's time loop -------------------------------------------
    def iterations(self, dt, maxiter, resid_out=None, iter0=0, ncellglob=None, nwrite=0, outdir=None):
        """The loop of iterations.f90:19-83 with its residual monitor every
        10 iterations (mod(iter,10)==1); returns the monitor rows
        (iter, ctime, RESIDNORM, divB).  With nwrite > 0 and an output
        directory, the Tecplot file (outdir/TEC/, when a plot mesh is set)
        and the restart file (outdir/) are queued after the iterations with
        mod(iter,nwrite)==1 and after the last one (iterations.f90:77-80),
        and written while the loop goes on."""
        import os
        rows = []
        ncg = ncellglob or self.ncell
        it = iter0
        if resid_out:
            with open(resid_out, "w") as f:
                f.write(" ITER    ctime     RESIDNORM   divB\n")
        if nwrite and outdir is not None and getattr(self, "_plot", None) is not None:
            os.makedirs(os.path.join(outdir, "TEC"), exist_ok=True)
        while True:
            it += 1
            self.rk_s5p3(dt, 1)
            if it % 10 == 1:
                m = self.monitor()
                rn = math.sqrt(m["residsum"] / (ncg * self.N * self.N * 9))
                db = math.sqrt(m["divbsum"] / (ncg * self.N * self.N))
                rows.append((it, self.maxima()["ctime"], rn, db))
                if resid_out:
                    with open(resid_out, "a") as f:
                        f.write(f" {it} {rows[-1][1]!r} {rn!r} {db!r}\n")
            last = it >= maxiter
            if nwrite and outdir is not None and (it % nwrite == 1 or last):
                from . import host
                if getattr(self, "_plot", None) is not None:
                    ct = self.maxima()["ctime"]
                    self.write_tecplot(os.path.join(outdir, "TEC", host.tecplot_filename(ct)))
                self.write_restart(os.path.join(outdir, host.restart_filename(it)), it)
            if last:
                break
        if nwrite and outdir is not None:
            self.output_wait()
        return rows
