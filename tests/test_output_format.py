"""CPU tests of the output row: the Tecplot plot mesh (tecplotter2dsetup)
from the host library against the oracle's restatement, the plot-node values
(tecplotter2d) of the oracle against a direct numpy evaluation, and the
restart / Tecplot files and names written by the host library against the
oracle's independent numpy restatement of the formats (write_data.f90,
tecplotter.f90:99-415), byte for byte."""
import numpy as np
import pytest

import sddc_oracle as O
from helpers import ALL_SMALL
from sddc_b200 import deck, host, mesh

MESHES = ["cylinder_n4", "channel_n3", "periodic_n4", "wallbox_vis1"]


@pytest.mark.parametrize("name", MESHES)
@pytest.mark.parametrize("nre", [1, 2, 3, 5])
def test_plot_mesh_matches_oracle(name, nre):
    m, t, ph, Q = ALL_SMALL[name]()
    pm = host.plot_mesh(m, nre)
    n, nc, px, gn, gf, cn = O.plot_setup(t.ivcell, m.xv, m.yv, t.IF2C, nre)
    assert (pm.plotnodes, pm.plotcells) == (n, nc)
    assert np.array_equal(pm.plotx, px)
    assert np.array_equal(pm.gnumnode, gn)
    assert np.array_equal(pm.gnode_factor, gf)
    assert np.array_equal(pm.connec, cn)
    # vertices, then nre-1 nodes per face, then (nre-1)^2 per cell
    assert n == m.nvert + t.nface * (nre - 1) + m.ncell * (nre - 1) ** 2
    assert nc == nre * nre * m.ncell
    # gnode_factor counts the cells whose plot points land on the node
    assert np.array_equal(np.bincount(gn.ravel(order="F"), minlength=n + 1)[1:], gf)
    # the first NVERT nodes are the mesh vertices
    assert np.array_equal(px[0, :m.nvert], m.xv) and np.array_equal(px[1, :m.nvert], m.yv)


def test_plot_mesh_rejects_unused_vertex():
    m = mesh.channel_box(3, 2)
    m.xv = np.append(m.xv, 9.0)
    m.yv = np.append(m.yv, 9.0)
    with pytest.raises(host.HostError, match="to no cell"):
        host.plot_mesh(m, 2)


def _numpy_plot_eval(N, Q, muAV, nre, gn, gf, Xs):
    """tecplotter2d by numpy (sums in a different order: within rounding)."""
    def h(i, x):
        return np.prod([(x - Xs[s]) / (Xs[i] - Xs[s]) for s in range(N) if s != i])
    pts = np.arange(nre + 1) / nre
    H = np.array([[h(i, x) for i in range(N)] for x in pts])  # (nre+1, N)
    n = gf.shape[0]
    acc = np.zeros((9, n))
    av = np.zeros((2, n))
    for c in range(Q.shape[3]):
        vals = np.einsum("kij,ai,bj->kab", Q[:, :, :, c], H, H)  # (9, ii, jj)
        for jj in range(nre + 1):
            for ii in range(nre + 1):
                g = gn[ii, jj, c] - 1
                acc[:, g] += vals[:, ii, jj]
                av[:, g] += muAV[:, c]
    Qs = acc / gf
    rho = Qs[0]
    u, v, w = Qs[1] / rho, Qs[2] / rho, Qs[3] / rho
    p = (Qs[4] - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (Qs[5] ** 2 + Qs[6] ** 2 + Qs[7] ** 2)) * (2.0 / 3.0)
    return np.array([rho, u, v, w, p, Qs[5], Qs[6], Qs[7], Qs[8]]), av / gf


@pytest.mark.parametrize("name,nre", [("cylinder_n4", 3), ("channel_n3", 2), ("periodic_n4", 4)])
def test_oracle_plot_eval_against_numpy(name, nre):
    m, t, ph, Q = ALL_SMALL[name]()
    pm = host.plot_mesh(m, nre)
    rng = np.random.default_rng(7)
    mu = rng.uniform(0, 1e-2, (2, m.ncell))
    pq, pa = O.plot_eval(t.N, Q, mu, nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    eq, ea = _numpy_plot_eval(t.N, Q, mu, nre, pm.gnumnode, pm.gnode_factor, t.Xs)
    assert np.allclose(pq, eq, rtol=1e-12, atol=1e-13)
    assert np.allclose(pa, ea, rtol=1e-12, atol=1e-16)
    # without muAV the plot's muAV and etaAV are 0
    pq0, pa0 = O.plot_eval(t.N, Q, None, nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    assert np.array_equal(pq0, pq) and not pa0.any()


def test_plot_eval_continuous_field_is_node_exact():
    """A state whose conserved variables are bilinear in x, y on a
    parallelogram mesh is reproduced exactly at shared nodes (every cell
    interpolates the same value there), so the node average is that value."""
    m = mesh.channel_box(4, 3, jitter=0.0)
    N, nre = 4, 3
    t = host.build_tables(m, N)
    x, y = t.xxsolu[0], t.xxsolu[1]
    Q = np.zeros((9, N, N, m.ncell), order="F")
    Q[0] = 1.0 + 0.1 * x + 0.05 * y
    Q[4] = 3.0 + 0.2 * x * y
    Q[5] = 0.3 - 0.1 * y
    pm = host.plot_mesh(m, nre)
    pq, _ = O.plot_eval(N, Q, None, nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    X, Y = pm.plotx
    assert np.allclose(pq[0], 1.0 + 0.1 * X + 0.05 * Y, rtol=1e-13)
    assert np.allclose(pq[5], 0.3 - 0.1 * Y, atol=1e-13)


@pytest.mark.parametrize("ctime,name", [
    (0.0, "TEC0000000.000.plt"), (1.25, "TEC0000001.250.plt"), (12.3456, "TEC0000012.346.plt"),
    (0.0625, "TEC0000000.063.plt"),    # an exact tie rounds away from zero
    (1.9996, "TEC0000001.000.plt"),    # the fraction rounds up to 1: the reference's name keeps int(ctime)
    (1234567.0005, "TEC1234567.001.plt"),
])
def test_tecplot_filename(ctime, name):
    assert host.tecplot_filename(ctime) == name
    assert O.tecplot_name(ctime) == name


def test_filenames_against_oracle():
    rng = np.random.default_rng(3)
    for ct in rng.uniform(0, 500, 200):
        assert host.tecplot_filename(ct) == O.tecplot_name(ct)
    for it in (0, 1, 11, 99999999, 12345678):
        assert host.restart_filename(it) == O.restart_name(it)
    assert host.restart_filename(7) == "restart.00000007.dat"


@pytest.mark.parametrize("name", ["cylinder_n4", "channel_n5"])
def test_restart_file_bytes_and_round_trip(tmp_path, name):
    m, t, ph, Q = ALL_SMALL[name]()
    p = tmp_path / "r.dat"
    host.restart_write(p, Q, 41, 0.123456789)
    data = p.read_bytes()
    assert data == O.restart_bytes(41, 0.123456789, Q)
    assert len(data) == 12 + m.ncell * (4 + 8 * 9 * t.N * t.N)
    Q2, it, ct = host.restart_read(p, t.N, m.ncell)
    assert (it, ct) == (41, 0.123456789) and np.array_equal(Q2, Q)
    # the Python deck helpers read and write the same file
    Q3, it3, ct3 = deck.read_restart(str(p), t.N, m.ncell)
    assert np.array_equal(Q3, Q) and (it3, ct3) == (41, 0.123456789)
    deck.write_restart(str(tmp_path / "d.dat"), Q, 41, 0.123456789)
    assert (tmp_path / "d.dat").read_bytes() == data


def test_restart_global_numbers(tmp_path):
    """IC2ICG on write and ICG2IC on read (read_data_restart.f90:53-62):
    records are placed by global number; unmapped records are skipped."""
    m, t, ph, Q = ALL_SMALL["channel_n3"]()
    nc = m.ncell
    rng = np.random.default_rng(5)
    icg = rng.permutation(nc).astype(np.int32) + 1
    p = tmp_path / "g.dat"
    host.restart_write(p, Q, 3, 1.5, icg=icg)
    assert p.read_bytes() == O.restart_bytes(3, 1.5, Q, icg)
    # a rank holding the cells in global order
    icg2ic = np.zeros(nc, np.int32)
    icg2ic[icg - 1] = np.arange(1, nc + 1)
    Q2, _, _ = host.restart_read(p, t.N, nc, icg2ic=icg2ic)
    assert np.array_equal(Q2, Q)
    # a rank holding only the first half of the global cells
    half = nc // 2
    sub = np.zeros(nc, np.int32)
    sub[:half] = np.arange(1, half + 1)
    Q3, _, _ = host.restart_read(p, t.N, half, nrec=nc, icg2ic=sub)
    order = np.argsort(icg)  # local cell holding global g is order[g-1]
    assert np.array_equal(Q3, Q[:, :, :, order[:half]])


def test_restart_short_file(tmp_path):
    m, t, ph, Q = ALL_SMALL["channel_n3"]()
    p = tmp_path / "s.dat"
    host.restart_write(p, Q, 1, 0.0)
    p.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(host.HostError, match="file ends before"):
        host.restart_read(p, t.N, m.ncell)
    with pytest.raises(host.HostError, match="cannot open"):
        host.restart_read(tmp_path / "missing.dat", t.N, m.ncell)


@pytest.mark.parametrize("name,nre", [("cylinder_n4", 3), ("periodic_n4", 1), ("wallbox_vis1", 4)])
def test_tecplot_file_bytes(tmp_path, name, nre):
    m, t, ph, Q = ALL_SMALL[name]()
    pm = host.plot_mesh(m, nre)
    rng = np.random.default_rng(11)
    mu = rng.uniform(0, 1e-3, (2, m.ncell))
    pq, pa = O.plot_eval(t.N, Q, mu, nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    p = tmp_path / "a.plt"
    host.tecplot_write(p, 0.75, pm, pq, pa)
    assert p.read_bytes() == O.tecplot_bytes(0.75, pm.plotx, pq, pa, pm.connec)
    # no AV: zeros
    host.tecplot_write(p, 0.75, pm, pq, None)
    assert p.read_bytes() == O.tecplot_bytes(0.75, pm.plotx, pq, None, pm.connec)


def test_tecplot_file_layout(tmp_path):
    """Reads the file back field by field (the reader a Tecplot user has)."""
    m, t, ph, Q = ALL_SMALL["channel_n3"]()
    pm = host.plot_mesh(m, 2)
    pq, pa = O.plot_eval(t.N, Q, None, 2, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    p = tmp_path / "b.plt"
    host.tecplot_write(p, 2.5, pm, pq, pa)
    b = p.read_bytes()
    assert b[:8] == b"#!TDV111"
    ints = np.frombuffer(b[8:16], "<i4")
    assert list(ints) == [1, 0]
    off = 16

    def read_string(off):
        chars = []
        while True:
            c = int(np.frombuffer(b[off:off + 4], "<i4")[0])
            off += 4
            if c == 0:
                return "".join(chars), off
            chars.append(chr(c))

    title, off = read_string(off)
    assert title == "step data"
    nvar = int(np.frombuffer(b[off:off + 4], "<i4")[0])
    off += 4
    names = []
    for _ in range(nvar):
        s, off = read_string(off)
        names.append(s)
    assert names == ["X", "Y", "RHO", "U", "V", "W", "P", "Bx", "By", "Bz", "Az", "muAV", "etaAV"]
    assert np.frombuffer(b[off:off + 4], "<f4")[0] == 299.0
    zone, off = read_string(off + 4)
    assert zone == "ZONE 001"
    off += 8
    assert np.frombuffer(b[off:off + 8], "<f8")[0] == 2.5
    off += 8
    zi = np.frombuffer(b[off:off + 48], "<i4")
    assert list(zi[:6]) == [-1, 3, 0, 0, 0, 0] and zi[6] == pm.plotnodes and zi[7] == pm.plotcells
    off += 48 + 8 + 4 * (nvar + 3)
    mm = np.frombuffer(b[off:off + 16 * nvar], "<f8").reshape(nvar, 2)
    off += 16 * nvar
    data = np.frombuffer(b[off:off + 4 * nvar * pm.plotnodes], "<f4").reshape(nvar, pm.plotnodes)
    off += 4 * nvar * pm.plotnodes
    assert np.array_equal(data[2], pq[0].astype(np.float32))
    assert mm[2, 0] == pq[0].min() and mm[2, 1] == pq[0].max()
    conn = np.frombuffer(b[off:], "<i4").reshape(pm.plotcells, 4)
    assert np.array_equal(conn, pm.connec.T - 1)
