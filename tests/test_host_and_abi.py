"""CPU tests of the host side: the C ABI libraries load and export what
include/*.h declares, the set-up tables are consistent, and the reference's
file formats round-trip."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from sddc_b200 import _native, cases, deck, host, mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(sddc_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_host_library_exports_header():
    syms = exported_symbols(_native.HOST_LIB)
    for name in declared_functions("sddc_host.h"):
        assert name in syms, name
    lib = ctypes.CDLL(_native.HOST_LIB)
    for name in declared_functions("sddc_host.h"):
        getattr(lib, name)


def test_gpu_library_exports_header():
    """libsddc_b200.so loads without a GPU and exports every sddc.h entry
    point (no compute call is made here)."""
    if not os.path.exists(_native.GPU_LIB):
        pytest.skip("libsddc_b200.so not built (run python -m sddc_b200.build)")
    syms = exported_symbols(_native.GPU_LIB)
    names = declared_functions("sddc.h")
    assert "sddc_rk_step" in names and "sddc_compresid" in names
    for name in names:
        assert name in syms, name
    lib = ctypes.CDLL(_native.GPU_LIB)
    for name in names:
        getattr(lib, name)


@pytest.mark.parametrize("maker", [
    lambda: mesh.cylinder_ogrid(6, 12),
    lambda: mesh.periodic_box(5, 4),
    lambda: mesh.channel_box(5, 4, jitter=0.2),
])
def test_every_cell_face_is_covered_once(maker):
    m = maker()
    t = host.build_tables(m, 4)
    nc = m.ncell
    seen = np.zeros((nc, 4), int)
    F = t.IF2C
    for f in t.ibfinter:
        l, r, lfl, lfr = F[f - 1]
        assert l < r  # the lower cell index visits the face first (left cell)
        seen[l - 1, lfl - 1] += 1
        seen[r - 1, lfr - 1] += 1
    for k1, k2 in t.cyc2fpair:
        seen[F[k1 - 1, 0] - 1, F[k1 - 1, 2] - 1] += 1
        seen[F[k2 - 1, 0] - 1, F[k2 - 1, 2] - 1] += 1
    for lst in (t.ibfinl, t.ibfout, t.ibfwal, t.ibfsymp, t.ibfree):
        for f in lst:
            seen[F[f - 1, 0] - 1, F[f - 1, 2] - 1] += 1
    assert np.all(seen == 1)
    assert t.counts["nreversed"] == 0
    assert t.Jac.min() > 0


def test_cylinder_boundaries():
    m = mesh.cylinder_ogrid(8, 16)
    t = host.build_tables(m, 4)
    c = t.counts
    assert c["nwall"] == 16 and c["ninlet"] + c["noutlet"] == 16 and c["ninlet"] == 8
    assert c["ninter"] == 2 * 8 * 16 - 16
    # radial grading keeps the 32-cell stretch
    assert abs(mesh.radial_ratio(256) ** 255 / (1.08 ** 31) - 1.0) < 0.1


def test_clockwise_cells_are_reversed_like_check_mesh():
    m = mesh.channel_box(3, 2)
    cw = m.ivcell[:, [1, 0, 3, 2]].copy()
    m2 = mesh.Mesh(m.xv, m.yv, cw, m.bnd_v, m.bnd_type)
    t = host.build_tables(m2, 3)
    assert t.counts["nreversed"] == m.ncell
    assert np.array_equal(t.ivcell, np.asfortranarray(m.ivcell))


def test_unlisted_boundary_face_is_an_error():
    m = mesh.channel_box(3, 3)
    keep = m.bnd_type != mesh.BC_CODE["FREE"]
    m2 = mesh.Mesh(m.xv, m.yv, m.ivcell, m.bnd_v[keep], m.bnd_type[keep])
    with pytest.raises(host.HostError, match="boundary condition"):
        host.build_tables(m2, 3)


def test_unpaired_cyclic_face_is_an_error():
    m = mesh.periodic_box(4, 4)
    m.dxcycl = 1.0  # wrong period: no partner matches
    with pytest.raises(host.HostError, match="partner"):
        host.build_tables(m, 3)


def test_mesh_files_round_trip(tmp_path):
    m = mesh.cylinder_ogrid(4, 8)
    p = m.write(str(tmp_path))
    m2 = mesh.Mesh.read(p["cel"], p["vrt"], p["bnd"])
    assert np.array_equal(m.ivcell, m2.ivcell)
    assert np.array_equal(m.xv, m2.xv) and np.array_equal(m.yv, m2.yv)
    assert np.array_equal(m.bnd_v, m2.bnd_v) and np.array_equal(m.bnd_type, m2.bnd_type)


def test_restart_and_deck_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    Q = np.asfortranarray(rng.standard_normal((9, 4, 4, 7)))
    path = str(tmp_path / "restart.dat")
    deck.write_restart(path, Q, iter_=12, ctime=0.5)
    assert os.path.getsize(path) == 4 + 8 + 7 * (4 + 8 * 9 * 16)
    Q2, it, ct = deck.read_restart(path, 4, 7)
    assert it == 12 and ct == 0.5 and np.array_equal(Q, Q2)
    d = deck.Deck(N=5, dt=1.25e-4, maxiter=2000, rinf=1.0, pinf=0.26666666666666666, bxinf=0.5)
    d.write(str(tmp_path / "QUAD.INP"))
    d2 = deck.Deck.read(str(tmp_path / "QUAD.INP"))
    assert d2 == d


def test_cases_initial_states():
    c = cases.config1()
    ph = c.physics
    assert abs(ph.pinf - 1.0 / (5.0 / 3.0 * 1.5 ** 2)) < 1e-15 and ph.bxinf == 0.5
    Q = c.initial_state()
    assert Q.shape == (9, 4, 4, 2048) and Q.flags.f_contiguous
    q0 = cases.conserved(1.0, 1.0, 0.0, 0.0, ph.pinf, 0.5, 0.0, 0.0, 0.0).ravel()
    assert np.abs(Q - q0[:, None, None, None]).max() <= 1e-6
    assert np.array_equal(Q, c.initial_state())  # seeded
