"""The discrete adjoint against the FP64 CPU tangent (the oracle built in
complex-step arithmetic) and against central finite differences.

* sddc_vjp_resid: <Qbar, V> = <Rbar, dR/dQ V> for random Rbar, V, on cases
  with every boundary kind; the c_h and free-stream adjoints likewise.
* sddc_adjoint_run: the gradient of the window-averaged drag/lift objective
  with respect to the initial field and the free stream, through several
  checkpoint segments, against the tangent of the oracle's own run."""
import numpy as np
import pytest

import sddc_oracle as O
from helpers import ALL_SMALL, case_cylinder, rel_l2
from sddc_b200 import cases
from sddc_b200.solver import Solver

H = 1e-30  # complex step


def _advance(t, ph, Q, dt, steps):
    """A state a few exact steps in (nonzero psi, running maxima, c_h > 0)."""
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q)
    s.rk_s5p3(dt, steps)
    Qn, mx = s.state()["Q"], s.maxima()
    s.close()
    return Qn, mx


def _fs(ph):
    return np.array([ph.rinf, ph.pinf, ph.uinf, ph.vinf, ph.bxinf, ph.byinf])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cylinder_n4", "channel_n3", "channel_n5", "periodic_n4", "wallbox_vis1",
                                  "wallbox_vis0"])
def test_vjp_resid_matches_tangent(name):
    m, t, ph, Q0 = ALL_SMALL[name]()
    dt = 0.5 * cases.cfl_dt(m, Q0, t.N)
    Q, mx = _advance(t, ph, Q0, dt, 3)
    rng = np.random.default_rng(7)
    lam = rng.standard_normal(Q.shape)
    V = rng.standard_normal(Q.shape) * np.abs(Q).max(axis=(1, 2, 3), keepdims=True)
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q, 0.0, mx["eigvmax"], mx["umax"])
    Qbar, par = s.vjp_resid(lam)
    s.close()
    # <lam, R'(Q) V> by the complex-step tangent of the oracle
    T = O.Oracle(t, ph, tangent=True)
    T.set_state(Q + 1j * H * V, 0.0, mx["eigvmax"], mx["umax"])
    T.compresid()
    jv = T.state()["resid"].imag / H
    a, b = float(np.vdot(lam, jv)), float(np.vdot(Qbar, V))
    assert abs(a - b) <= 1e-11 * (abs(np.vdot(np.abs(lam), np.abs(jv))) + 1e-300), (a, b)
    # the residual is affine in c_h: central difference in the running max
    o = O.Oracle(t, ph)
    L, U = mx["eigvmax"], mx["umax"]
    dl = 1e-3 * L
    o.set_state(Q, 0.0, L + dl, U)
    o.compresid()
    rp, cp = o.state()["resid"], o.maxima()["c_h"]
    o.set_state(Q, 0.0, L - dl, U)
    o.compresid()
    rm, cm = o.state()["resid"], o.maxima()["c_h"]
    cbar = float(np.vdot(lam, rp - rm)) / (cp - cm)
    assert abs(cbar - par[0]) <= 1e-8 * (abs(cbar) + np.abs(lam).sum() * 1e-3), (cbar, par[0])
    # the free stream through the boundary states
    fs = _fs(ph)
    for k in range(6):
        T.set_state(Q.astype(np.complex128), 0.0, L, U)
        e = np.zeros(6, dtype=np.complex128)
        e[k] = 1j * H
        T.set_freestream(fs + e)
        T.compresid()
        d = float(np.vdot(lam, T.state()["resid"].imag / H))
        assert abs(d - par[1 + k]) <= 1e-10 * (abs(d) + 1.0), (k, d, par[1 + k])
    T.set_freestream(fs.astype(np.complex128))


def _oracle_objective(t, ph, Q0, dt, nsteps, n1, n2, wd, wl, tangent=False, fs=None):
    """J of the oracle's own run (complex in tangent mode)."""
    o = O.Oracle(t, ph, tangent=tangent)
    if fs is not None:
        o.set_freestream(fs)
    o.set_state(Q0)
    w = O.sp_weights(O.operators(t.N)[0])
    U2 = ph.uinf ** 2 + ph.vinf ** 2
    dx, dy = ph.uinf / np.sqrt(U2), ph.vinf / np.sqrt(U2)
    norm = 2.0 / (ph.rinf * U2)
    J = 0.0
    for n in range(nsteps + 1):
        if n > 0:
            o.rk_s5p3(dt, 1)
        if n1 <= n <= n2:
            fx, fy = o.wall_force(w)
            J = J + wd * norm * (fx * dx + fy * dy) + wl * norm * (-fx * dy + fy * dx)
    return J / (n2 - n1 + 1), o


@pytest.mark.gpu
@pytest.mark.parametrize("wd,wl", [(1.0, 0.0), (0.3, -1.7)])
def test_adjoint_run_matches_tangent(wd, wl):
    m, t, ph, Q0 = case_cylinder(6, 12, 4, seed=5)
    dt = cases.cfl_dt(m, Q0, t.N)
    nsteps, n1, n2 = 12, 4, 12
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q0)
    r = s.adjoint_run(dt, nsteps, n1, n2, w_drag=wd, w_lift=wl, checkpoint_every=5)
    Qfin = s.state()["Q"]
    s.close()
    J0, o = _oracle_objective(t, ph, Q0, dt, nsteps, n1, n2, wd, wl)
    assert abs(r["J"] - J0) <= 1e-12 * max(abs(J0), 1.0)
    # the context ends at the oracle's (bit-equal) final state
    assert np.array_equal(Qfin, o.state()["Q"])
    rng = np.random.default_rng(11)
    for trial in range(3):
        V = rng.standard_normal(Q0.shape) * np.abs(Q0).max(axis=(1, 2, 3), keepdims=True)
        Jt, _ = _oracle_objective(t, ph, Q0 + 1j * H * V, dt, nsteps, n1, n2, wd, wl, tangent=True)
        d_tan = Jt.imag / H
        d_adj = float(np.vdot(r["Qbar0"], V))
        assert abs(d_tan - d_adj) <= 1e-9 * (abs(d_tan) + 1e-12), (trial, d_tan, d_adj)
    fs = _fs(ph)
    for k in (1, 4):  # pinf and bxinf: the inflow Mach and Alfven numbers
        e = np.zeros(6, dtype=np.complex128)
        e[k] = 1j * H
        Jt, _ = _oracle_objective(t, ph, Q0.astype(np.complex128), dt, nsteps, n1, n2, wd, wl, tangent=True,
                                  fs=fs + e)
        d_tan = Jt.imag / H
        assert abs(d_tan - r["parbar"][k]) <= 1e-9 * (abs(d_tan) + 1e-12), (k, d_tan, r["parbar"][k])


@pytest.mark.gpu
def test_adjoint_checkpoint_interval_is_bit_neutral():
    m, t, ph, Q0 = case_cylinder(5, 10, 4, seed=6)
    dt = cases.cfl_dt(m, Q0, t.N)
    out = []
    for k in (1, 4, 100):
        s = Solver(t, ph, precision="fp64_exact")
        s.set_state(Q0)
        out.append(s.adjoint_run(dt, 9, 0, 9, w_drag=1.0, w_lift=0.5, checkpoint_every=k))
        s.close()
    for r in out[1:]:
        assert r["J"] == out[0]["J"]
        assert np.array_equal(r["Qbar0"], out[0]["Qbar0"])
        assert np.array_equal(r["parbar"], out[0]["parbar"])


@pytest.mark.gpu
def test_adjoint_central_differences():
    """Central differences (h = 1e-6) of J through the GPU forward run."""
    m, t, ph, Q0 = case_cylinder(8, 16, 4, seed=8)
    dt = cases.cfl_dt(m, Q0, t.N)
    nsteps, n1, n2 = 30, 20, 30
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q0)
    r = s.adjoint_run(dt, nsteps, n1, n2, w_drag=1.0, w_lift=1.0)
    rng = np.random.default_rng(3)
    h = 1e-6
    for trial in range(4):
        V = rng.uniform(-1, 1, Q0.shape) * np.abs(Q0).max(axis=(1, 2, 3), keepdims=True)
        Js = []
        for sgn in (1, -1):
            s.set_state(Q0 + sgn * h * V)
            Js.append(s.adjoint_run(dt, nsteps, n1, n2, w_drag=1.0, w_lift=1.0, gradient=False)["J"])
        fd = (Js[0] - Js[1]) / (2 * h)
        ad = float(np.vdot(r["Qbar0"], V))
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-3), (trial, fd, ad)
    s.close()


def _cs_field(ms, ma, noise):
    """The cylinder free-stream field plus noise, in complex arithmetic."""
    p = 1.0 / (cases.GAMMA * ms * ms)
    bx = 1.0 / ma
    q = np.array([1.0, 1.0, 0.0, 0.0, p / (cases.GAMMA - 1.0) + 0.5 + 0.5 * bx * bx, bx, 0.0, 0.0, 0.0],
                 dtype=np.complex128)
    return np.asfortranarray(q[:, None, None, None] + noise), np.array([1.0, p, 1.0, 0.0, bx, 0.0],
                                                                       dtype=np.complex128)


@pytest.mark.gpu
def test_torch_function_mach_gradients():
    """dJ/dMs and dJ/dMA through the autograd wrapper (boundary states and
    initial field) against the complex-step tangent of the oracle's run."""
    from sddc_b200 import adjoint
    m, t, ph, _ = case_cylinder(6, 12, 4)
    ms, ma = 0.5, 2.0
    noise = np.random.default_rng(4).uniform(-1e-3, 1e-3, (9, t.N, t.N, t.ncell))
    Qr, _ = _cs_field(ms, ma, noise)
    dt = cases.cfl_dt(m, Qr.real.copy(order="F"), t.N)
    nsteps, n1, n2, wd, wl = 12, 4, 12, 1.0, 0.5
    prob = adjoint.DragLiftProblem(t, dt, nsteps, n1, n2, w_drag=wd, w_lift=wl, checkpoint_every=5)
    J, dms, dma, _ = adjoint.mach_gradients(prob, ms, ma, noise)
    prob.close()
    phys = cases.cylinder_physics(ms, ma)
    for which, ad in (("ms", dms), ("ma", dma)):
        Qc, fsc = _cs_field(ms + (1j * H if which == "ms" else 0), ma + (1j * H if which == "ma" else 0), noise)
        Jt, _ = _oracle_objective(t, phys, Qc, dt, nsteps, n1, n2, wd, wl, tangent=True, fs=fsc)
        assert abs(Jt.real - J) <= 1e-12 * abs(J)
        d_tan = Jt.imag / H
        assert abs(d_tan - ad) <= 1e-9 * (abs(d_tan) + 1e-12), (which, d_tan, ad)


@pytest.mark.gpu
def test_adjoint_long_run_matches_tangent():
    """200 steps on a 24x48 cylinder (hundreds of stages raise a running
    maximum): the adjoint equals the complex-step tangent to rounding."""
    import os
    O.set_threads(os.cpu_count() or 1)
    from sddc_b200 import host, mesh
    m = mesh.cylinder_ogrid(24, 48)
    t = host.build_tables(m, 4)
    ph = cases.cylinder_physics(ms=0.5, ma=2.0)
    Q0 = cases.freestream_state(ph, 4, m.ncell, noise=1e-6, seed=0)
    dt = cases.cfl_dt(m, Q0, 4)
    nsteps, n1 = 200, 150
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q0)
    r = s.adjoint_run(dt, nsteps, n1, nsteps, w_drag=1.0, w_lift=0.25)
    s.close()
    assert r["stats"]["owner_stages"] > 100
    V = np.random.default_rng(1).uniform(-1, 1, Q0.shape) * np.abs(Q0).max(axis=(1, 2, 3), keepdims=True)
    Jt, _ = _oracle_objective(t, ph, Q0 + 1j * H * V, dt, nsteps, n1, nsteps, 1.0, 0.25, tangent=True)
    d_tan, d_adj = Jt.imag / H, float(np.vdot(r["Qbar0"], V))
    assert abs(d_tan - d_adj) <= 1e-12 * abs(d_tan), (d_tan, d_adj)


@pytest.mark.gpu
def test_adjoint_fullsize_central_differences():
    """The configured adjoint case (cylinder 128x256, p = 3, C_D over steps
    1000-1200): 16 seeded directions of the initial field against central
    differences with h = 1e-9.  A 1e-6 step crosses kinks of the max-based
    c_h; at 1e-9 the rounding of J over 1200 steps (~1e-14 relative), over
    2h, bounds the difference quotient to ~1e-5 relative, so that is the
    check's resolution (the adjoint itself equals the tangent to rounding,
    test_adjoint_long_run_matches_tangent)."""
    from sddc_b200 import host, mesh
    m = mesh.cylinder_ogrid(128, 256)
    t = host.build_tables(m, 4)
    ph = cases.cylinder_physics(ms=0.5, ma=2.0)
    Q0 = cases.freestream_state(ph, 4, m.ncell, noise=1e-6, seed=0)
    dt = cases.cfl_dt(m, Q0, 4)
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q0)
    r = s.adjoint_run(dt, 1200, 1000, 1200, w_drag=1.0)
    rng = np.random.default_rng(16)
    scale = np.abs(Q0).max(axis=(1, 2, 3), keepdims=True)
    h, errs = 1e-9, []
    for _ in range(16):
        V = rng.uniform(-1, 1, Q0.shape) * scale
        js = []
        for sg in (1, -1):
            s.set_state(Q0 + sg * h * V)
            js.append(s.adjoint_run(dt, 1200, 1000, 1200, w_drag=1.0, gradient=False)["J"])
        ad = float(np.vdot(r["Qbar0"], V))
        errs.append(abs((js[0] - js[1]) / (2 * h) - ad) / abs(ad))
    s.close()
    assert max(errs) < 1e-4 and float(np.median(errs)) < 1e-5, errs
