"""Known-answer tests that pin the CPU oracle to the mathematics.

The reference ships no golden vectors and cannot be compiled here, so the
oracle is pinned by properties any correct spectral-difference MHD residual
must have: operator exactness, free-stream preservation, Rusanov
consistency, conservation on periodic domains, convergence order, RK order,
and equality of the skipped viscous chain at mu = eta0 = 0.
"""
import math

import numpy as np
import pytest

import sddc_oracle as O
from helpers import ALL_SMALL, case_channel, case_periodic, channel_physics, rel_l2
from sddc_b200 import cases, host, mesh


@pytest.mark.parametrize("N", [2, 3, 4, 5, 6])
def test_operators_exact_on_polynomials(N):
    Xs, Xf, L, M = O.operators(N)
    assert np.allclose(L.sum(axis=1), 1.0, atol=1e-13)          # interpolation of constants
    assert np.allclose(M.sum(axis=0), 0.0, atol=1e-11)          # derivative of constants
    for deg in range(N):                                         # degree <= N-1 interpolated exactly
        assert np.allclose(L @ Xs ** deg, Xf ** deg, atol=1e-12)
    for deg in range(N + 1):                                     # derivative of degree <= N from flux points
        d = deg * Xs ** (deg - 1) if deg else np.zeros(N)
        assert np.allclose(M.T @ Xf ** deg, d, atol=1e-10)
    assert Xf[0] == 0.0 and Xf[-1] == 1.0 and np.all(np.diff(Xf) > 0)
    assert np.all(np.diff(Xs) > 0) and np.allclose(Xs + Xs[::-1], 1.0)


def test_host_tables_equal_oracle_restatement():
    for N in (3, 4, 5):
        m = mesh.cylinder_ogrid(5, 9)
        t = host.build_tables(m, N)
        Xs, Xf, L, M = O.operators(N)
        assert np.array_equal(L, t.Lmat) and np.array_equal(M, t.Mmat)
        assert np.array_equal(Xs, t.Xs) and np.array_equal(Xf, t.Xf)
        S1, S2, J = O.metrics(N, t.ivcell, m.xv, m.yv)
        assert np.array_equal(S1, t.S1) and np.array_equal(S2, t.S2) and np.array_equal(J, t.Jac)
        assert J.min() > 0


@pytest.mark.parametrize("name", ["periodic", "channel", "cylinder"])
def test_freestream_preservation(name):
    N = 4
    if name == "periodic":
        m = mesh.periodic_box(6, 5)
        ph = cases.Physics(rinf=1.1, pinf=0.9, uinf=0.3, vinf=0.2, bxinf=0.5, byinf=0.1, dxcycl=2 * math.pi,
                           dycycl=2 * math.pi)
    elif name == "channel":
        m = mesh.channel_box(6, 5, jitter=0.25, sides=("FREE", "OUTL", "FREE", "INLE"))
        ph = channel_physics()
    else:
        m = mesh.cylinder_ogrid(6, 12)
        ph = cases.cylinder_physics(0.5, 2.0)
    t = host.build_tables(m, N)
    Q = cases.freestream_state(ph, N, m.ncell, noise=0.0)
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.compresid()
    r = o.state()["resid"]
    if name == "cylinder":
        # the wall ghost state is not the free stream: only cells away from
        # the wall ring preserve it
        r = r[..., 2 * 12:]
    assert np.abs(r).max() < 1e-11


def test_rusanov_consistency():
    rng = np.random.default_rng(0)
    for _ in range(20):
        q = cases.conserved(rng.uniform(0.5, 2), *rng.uniform(-1, 1, 3), rng.uniform(0.5, 2),
                            *rng.uniform(-1, 1, 3), rng.uniform(-0.1, 0.1)).ravel()
        nf = rng.uniform(-2, 2, 2)
        c_h = rng.uniform(0, 2)
        for sl in (1, -1):
            Fl, Fr, eig, _ = O.point_rusanov(q, q, nf, sign_l=sl, sign_r=-1, c_h=c_h)
            F, G, _ = O.point_iflux(q, c_h)
            # F(Q,Q) is the physical flux projected on the (unnormalised) normal
            assert np.allclose(Fl, F * nf[0] + G * nf[1], rtol=1e-12, atol=1e-12)
            assert np.array_equal(Fr, -sl * Fl)
            assert eig > 0


def test_conservation_periodic():
    m, t, ph, Q = case_periodic(n=6, N=4)
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.compresid()
    r = o.state()["resid"]
    Xs = t.Xs
    V = np.vander(Xs, increasing=True).T
    w = np.linalg.solve(V, 1.0 / np.arange(1, len(Xs) + 1))
    wij = w[:, None] * w[None, :]
    # density has no source: its integral is conserved to round-off
    total = np.sum(r[0] * t.Jac * wij[..., None])
    scale = np.sum(np.abs(r[0]) * t.Jac * wij[..., None])
    assert abs(total) < 1e-12 * max(scale, 1.0)


def test_divergence_free_linear_field_has_no_source():
    # B = (y, x) is divergence free and lies in the SD space: divB == 0
    m = mesh.channel_box(4, 3, jitter=0.2, sides=("FREE",) * 4)
    N = 4
    t = host.build_tables(m, N)
    x, y = t.xxsolu[0], t.xxsolu[1]
    Q = np.asfortranarray(cases.conserved(np.ones_like(x), 0.1, 0.2, 0.0, 1.0, 0.3 * y, 0.3 * x, 0.0, 0.0))
    o = O.Oracle(t, channel_physics())
    o.set_state(Q)
    o.compresid()
    g = o.state()["nablaQs"]
    divB = g[5, 0] + g[6, 1]
    assert np.abs(divB).max() < 1e-12
    assert np.allclose(g[5, 1], 0.3, atol=1e-12) and np.allclose(g[6, 0], 0.3, atol=1e-12)


def test_convergence_order_smooth_wave():
    """Advected density wave on a periodic box converges at about order N."""
    N = 4
    errs = []
    for n in (4, 8):
        m = mesh.periodic_box(n, n)
        t = host.build_tables(m, N)
        ph = cases.Physics(rinf=1, pinf=1, uinf=1, vinf=0.5, dxcycl=2 * np.pi, dycycl=2 * np.pi)

        def wave(tt):
            xx, yy = t.xxsolu[0] - 1.0 * tt, t.xxsolu[1] - 0.5 * tt
            return np.asfortranarray(cases.conserved(1 + 0.2 * np.sin(xx + yy), 1.0, 0.5, 0.0, 1.0, 0.3, 0.2, 0.0, 0.0))

        T = 0.25
        ns = int(math.ceil(T / (0.1 * (2 * np.pi / n) / (N * 3.0))))
        o = O.Oracle(t, ph)
        o.set_state(wave(0.0))
        o.rk_s5p3(T / ns, ns)
        errs.append(np.sqrt(np.mean((o.state()["Q"][0] - wave(T)[0]) ** 2)))
    assert math.log2(errs[0] / errs[1]) > 3.0


def test_rk_s5p3_third_order():
    lam = -1.0 + 0.5j
    errs = []
    for n in (20, 40):
        dt = 1.0 / n
        y = np.array([1.0, 0.0])  # (re, im)

        def rhs(v):
            z = (v[0] + 1j * v[1]) * lam
            return np.array([z.real, z.imag])

        for _ in range(n):
            qk0 = y.copy()
            q = y.copy()
            qka = None
            for stage in range(1, 6):
                r = rhs(q)
                q = O.rk_s5p3_combine(stage, dt, q, qk0, qka if qka is not None else q, r)
                if stage == 2:
                    qka = q.copy()
            y = q
        errs.append(abs((y[0] + 1j * y[1]) - np.exp(lam)))
    assert math.log2(errs[0] / errs[1]) > 2.8


@pytest.mark.parametrize("name", ["cylinder_n4", "channel_n4", "periodic_n4", "wallbox_vis1"])
def test_skipping_the_ideal_viscous_chain_is_exact(name):
    """With mu = eta0 = 0 the viscous chain adds exactly +0.0 to the residual:
    the oracle's full chain and the skipped chain agree bit for bit."""
    m, t, ph, Q = ALL_SMALL[name]()
    full = O.Oracle(t, ph, skip_ideal_viscous=False)
    skip = O.Oracle(t, ph, skip_ideal_viscous=True)
    for o in (full, skip):
        o.set_state(Q)
        o.rk_s5p3(1e-3, 2)
        o.compresid()
    a, b = full.state(), skip.state()
    assert np.array_equal(a["Q"], b["Q"])
    assert np.array_equal(a["resid"], b["resid"])
    assert np.array_equal(a["nablaQs"], b["nablaQs"])
    assert np.array_equal(a["sm_ind"], b["sm_ind"], equal_nan=True)
    fa = full.fluxes()
    assert np.all(fa["Fv1"] == 0.0) and np.all(fa["Gv2"] == 0.0)


def test_oracle_threads_do_not_change_results():
    m, t, ph, Q = case_channel(N=4)
    out = []
    for nth in (1, 4):
        O.set_threads(nth)
        o = O.Oracle(t, ph)
        o.set_state(Q)
        o.rk_s5p3(1e-3, 3)
        out.append(o.state()["Q"])
    O.set_threads(1)
    assert np.array_equal(out[0], out[1])


def test_five_stage_rk_matches_s5p3_on_smooth_case():
    m, t, ph, Q = case_periodic(N=4)
    a, b = O.Oracle(t, ph), O.Oracle(t, ph)
    a.set_state(Q)
    b.set_state(Q)
    a.rk_s5p3(2e-3, 5)
    b.five_stage_rk(2e-3, 5)
    assert rel_l2(a.state()["Q"], b.state()["Q"]) < 1e-6


def test_time_integrators_reach_their_order():
    """Self-convergence in time on a smooth periodic wave.  The runs share the
    mesh, so the spatial error cancels: FiveStageRk (iterations.f90:88-156)
    converges at fourth order, RK_S5P3 (iterations.f90:158-213) at third, on
    the full residual.  B = psi = 0 removes every c_h term, and a uniform
    flow keeps the face-normal velocities away from the kink of |Vn|, so the
    right-hand side is smooth."""
    m = mesh.periodic_box(4, 4)
    t = host.build_tables(m, 4)
    ph = cases.Physics(rinf=1.0, pinf=1.0, uinf=0.8, vinf=0.5, bxinf=0.0, byinf=0.0, dxcycl=2 * math.pi,
                       dycycl=2 * math.pi)
    x, y = t.xxsolu[0], t.xxsolu[1]
    z = 0.0 * x
    Q = np.asfortranarray(cases.conserved(1 + 0.1 * np.sin(x) * np.cos(y), 0.8 + z, 0.5 + z, z,
                                          1 + 0.05 * np.cos(x + y), z, z, z, z))
    T = 0.2

    def run(method, n):
        o = O.Oracle(t, ph, skip_ideal_viscous=True)
        o.set_state(Q)
        getattr(o, method)(T / n, n)
        return o.state()["Q"]

    for method, order in (("five_stage_rk", 4), ("rk_s5p3", 3)):
        ref = run(method, 256)
        e = [np.linalg.norm(run(method, n) - ref) for n in (8, 16, 32)]
        for k in range(2):
            assert math.log2(e[k] / e[k + 1]) > order - 0.2, (method, e)
