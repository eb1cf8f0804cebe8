"""CPU tests of the 8-node (serendipity) cells of CURVE_WALL = 1: the host
library's metrics against the oracle's restatement of MAPDER_8_NODE and
calcjacob (bit for bit), known answers (straight mid-side nodes give the
bilinear map, arcs converge to the annulus area, the curved metrics keep a
uniform state steady), the 8-node file format and the curved plot mesh."""
import math

import numpy as np
import pytest

import sddc_oracle as O
from helpers import wavy_periodic_box
from sddc_b200 import cases, host, mesh


@pytest.mark.parametrize("N", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("which", ["cylinder", "wavy"])
def test_metrics8_match_oracle(N, which):
    m = mesh.cylinder_ogrid(6, 12, curved=True) if which == "cylinder" else wavy_periodic_box(5)
    t = host.build_tables(m, N)
    S1, S2, J = O.metrics8(N, m.xxf_cell)
    assert np.array_equal(t.S1, S1) and np.array_equal(t.S2, S2) and np.array_equal(t.Jac, J)
    assert t.Jac.min() > 0


def test_straight_midpoints_give_the_bilinear_map():
    m = mesh.channel_box(4, 3, jitter=0.2, seed=3)
    m8 = mesh.channel_box(4, 3, jitter=0.2, seed=3)
    m8.xxf_cell = mesh.eight_node_cells(m8)
    for N in (3, 5):
        a, b = host.build_tables(m, N), host.build_tables(m8, N)
        for k in ("S1", "S2", "Jac", "xxsolu"):
            assert np.allclose(getattr(a, k), getattr(b, k), rtol=0, atol=1e-14), k


def test_arcs_converge_to_the_annulus_area():
    exact = math.pi * (20.0 ** 2 - 0.5 ** 2)
    errs = {}
    for nt in (12, 24):
        for curved in (False, True):
            m = mesh.cylinder_ogrid(6, nt, curved=curved)
            t = host.build_tables(m, 4)
            w = O.sp_weights(t.Xs)
            errs[nt, curved] = abs(float(np.einsum("i,j,ijc->", w, w, t.Jac)) - exact)
    # chords lose O(h^2) of the area, quadratic arcs O(h^4)
    assert errs[12, True] < 1e-2 * errs[12, False]
    assert errs[12, True] / errs[24, True] > 12.0
    assert errs[12, False] / errs[24, False] > 3.5


@pytest.mark.parametrize("N", [3, 4, 5])
def test_uniform_state_stays_steady_on_curved_cells(N):
    """Freestream preservation: the SD divergence of the quadratic metric
    terms vanishes, so a uniform state on periodic curved cells has a
    residual at rounding level."""
    m = wavy_periodic_box(6)
    t = host.build_tables(m, N)
    ph = cases.Physics(rinf=1.0, pinf=1.0, uinf=0.3, vinf=-0.2, bxinf=0.4, byinf=0.1, dxcycl=2 * math.pi,
                       dycycl=2 * math.pi)
    Q = cases.freestream_state(ph, N, m.ncell, noise=0.0, seed=0)
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.compresid()
    assert np.abs(o.state()["resid"]).max() < 1e-10


def test_solution_points_lie_on_the_8_node_map():
    m = mesh.cylinder_ogrid(4, 8, curved=True)
    t = host.build_tables(m, 3)
    # a cell of the first ring: its wall-side solution points sit on the map,
    # between the arc and the chord
    r = np.hypot(t.xxsolu[0], t.xxsolu[1])
    assert r.min() > 0.5


def test_vrt8_file_round_trip(tmp_path):
    m = mesh.cylinder_ogrid(4, 8, curved=True)
    paths = m.write(str(tmp_path))
    assert len(open(paths["vrt8"]).read().splitlines()) == 8 * m.ncell
    m2 = mesh.Mesh.read(paths["cel"], paths["vrt"], paths["bnd"], vrt8=paths["vrt8"])
    assert m2.curved and np.array_equal(m2.xxf_cell, m.xxf_cell)
    t1, t2 = host.build_tables(m, 4), host.build_tables(m2, 4)
    assert np.array_equal(t1.Jac, t2.Jac) and np.array_equal(t1.S1, t2.S1)


@pytest.mark.parametrize("nre", [2, 3, 4])
def test_curved_plot_mesh_matches_oracle(nre):
    m = mesh.cylinder_ogrid(6, 12, curved=True)
    t = host.build_tables(m, 4)
    pm = host.plot_mesh(m, nre)
    n, nc, px, gn, gf, cn = O.plot_setup(t.ivcell, m.xv, m.yv, t.IF2C, nre, m.xxf_cell)
    assert (pm.plotnodes, pm.plotcells) == (n, nc)
    assert np.array_equal(pm.plotx, px) and np.array_equal(pm.gnumnode, gn)
    assert np.array_equal(pm.gnode_factor, gf) and np.array_equal(pm.connec, cn)
    # the plot nodes of the wall follow the quadratic arc: within its
    # interpolation error of the circle, far closer than the chords
    rr = np.hypot(px[0], px[1])
    wall = np.abs(rr - 0.5) < 0.02
    assert np.abs(rr[wall] - 0.5).max() < 1e-4
    pb = host.plot_mesh(mesh.cylinder_ogrid(6, 12), nre)
    rb = np.hypot(pb.plotx[0], pb.plotx[1])
    assert np.abs(rb[np.abs(rb - 0.5) < 0.02] - 0.5).max() > 1e-3
