"""Restart and Tecplot output from the device state, through the C ABI
(sddc_set_plot, sddc_plot_nodes, sddc_write_tecplot, sddc_write_restart,
sddc_output_wait), against the oracle: the plot-node values of tecplotter2d
bit for bit (every form evaluates them in exact FP64), the files byte for
byte, and the background writes isolated from the steps that follow them."""
import os

import numpy as np
import pytest

import sddc_oracle as O
from helpers import ALL_SMALL
from sddc_b200 import cases, host
from sddc_b200.solver import EIO, SddcError, Solver

pytestmark = pytest.mark.gpu


def _stepped(name, precision, steps=3):
    m, t, ph, Q = ALL_SMALL[name]()
    s = Solver(t, ph, precision=precision)
    s.set_state(Q)
    dt = 0.2 * cases.cfl_dt(m, Q, t.N)
    s.rk_s5p3(dt, steps)
    return m, t, ph, s, dt


@pytest.mark.parametrize("name,nre", [("cylinder_n4", 3), ("channel_n5", 2), ("periodic_n4", 4),
                                      ("wallbox_vis1", 1)])
@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "mixed"])
def test_plot_nodes_bit_exact(name, nre, precision):
    m, t, ph, s, _ = _stepped(name, precision)
    pm = host.plot_mesh(m, nre)
    s.set_plot(pm)
    pq, pa = s.plot_nodes()
    st = s.state(muAV=ph.vismode == 1 and ph.artiv == 1)
    mu = st.get("muAV")
    eq, ea = O.plot_eval(t.N, st["Q"], mu, nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    assert np.array_equal(pq, eq)
    assert np.array_equal(pa, ea)
    if mu is None:
        assert not pa.any()
    s.close()


@pytest.mark.parametrize("name,nre", [("cylinder_n4", 3), ("wallbox_vis1", 2)])
def test_tecplot_file_bytes(tmp_path, name, nre):
    m, t, ph, s, _ = _stepped(name, "fp64")
    pm = host.plot_mesh(m, nre)
    s.set_plot(pm)
    p = tmp_path / "x.plt"
    s.write_tecplot(p)
    s.output_wait()
    st = s.state(muAV=ph.vismode == 1 and ph.artiv == 1)
    ct = s.maxima()["ctime"]
    eq, ea = O.plot_eval(t.N, st["Q"], st.get("muAV"), nre, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
    assert p.read_bytes() == O.tecplot_bytes(ct, pm.plotx, eq, ea, pm.connec)
    s.close()


@pytest.mark.parametrize("precision", ["fp64_exact", "mixed"])
def test_restart_file_round_trip(tmp_path, precision):
    m, t, ph, s, dt = _stepped("cylinder_n5", precision, steps=4)
    p = tmp_path / "r.dat"
    icg = np.arange(m.ncell, 0, -1, dtype=np.int32)
    s.write_restart(p, 4, icg=icg)
    s.output_wait()
    st = s.state()
    ct = s.maxima()["ctime"]
    assert p.read_bytes() == O.restart_bytes(4, ct, st["Q"], icg)
    icg2ic = np.zeros(m.ncell, np.int32)
    icg2ic[icg - 1] = np.arange(1, m.ncell + 1)
    Q2, it, ct2 = host.restart_read(p, t.N, m.ncell, icg2ic=icg2ic)
    assert it == 4 and ct2 == ct and np.array_equal(Q2, st["Q"])
    s.close()
    if precision == "fp64_exact":
        # a run restarted from the file (initsetup.f90:156-158: the running
        # maxima start again from 0, initsetup.f90:166-167) against the oracle
        # restarted from the same file
        r = Solver(t, ph, precision=precision)
        o = O.Oracle(t, ph)
        r.set_state(Q2, ct2)
        o.set_state(Q2, ct2)
        r.rk_s5p3(dt, 2)
        o.rk_s5p3(dt, 2)
        assert np.array_equal(r.state()["Q"], o.state()["Q"])
        r.close()


def test_writes_are_snapshots(tmp_path):
    """Files queued before further steps hold the state at the write call,
    and the steps are the same as without output."""
    m, t, ph, Q = ALL_SMALL["cylinder_n4"]()
    dt = 0.2 * cases.cfl_dt(m, Q, t.N)
    pm = host.plot_mesh(m, 3)
    a = Solver(t, ph, precision="fp64")
    b = Solver(t, ph, precision="fp64")
    a.set_state(Q)
    b.set_state(Q)
    b.set_plot(pm)
    snaps = []
    for k in range(3):
        a.rk_s5p3(dt, 2)
        b.rk_s5p3(dt, 2)
        snaps.append(b.state()["Q"].copy())
        b.write_restart(tmp_path / f"r{k}.dat", k)
        b.write_tecplot(tmp_path / f"t{k}.plt")
        b.rk_s5p3(dt, 1)  # steps while the files are written
        a.rk_s5p3(dt, 1)
    b.output_wait()
    assert np.array_equal(a.state()["Q"], b.state()["Q"])
    for k in range(3):
        Qk, it, _ = host.restart_read(tmp_path / f"r{k}.dat", t.N, m.ncell)
        assert it == k and np.array_equal(Qk, snaps[k])
        eq, _ = O.plot_eval(t.N, snaps[k], None, 3, pm.plotnodes, pm.gnumnode, pm.gnode_factor)
        data = (tmp_path / f"t{k}.plt").read_bytes()
        rho = np.frombuffer(data, "<f4", count=pm.plotnodes, offset=len(data) - 4 * 4 * pm.plotcells
                            - 4 * 11 * pm.plotnodes)
        assert np.array_equal(rho, eq[0].astype(np.float32))
    a.close()
    b.close()


def test_iterations_write_schedule(tmp_path):
    """iterations.f90:77-80: output after mod(iter,nwrite)==1 and the last
    iteration, named by iteration and solution time."""
    m, t, ph, Q = ALL_SMALL["channel_n3"]()
    dt = 0.2 * cases.cfl_dt(m, Q, t.N)
    s = Solver(t, ph, precision="fp64")
    s.set_state(Q)
    s.set_plot(host.plot_mesh(m, 2))
    s.iterations(dt, 25, nwrite=10, outdir=str(tmp_path))
    restarts = sorted(f for f in os.listdir(tmp_path) if f.startswith("restart."))
    assert restarts == ["restart.00000001.dat", "restart.00000011.dat", "restart.00000021.dat",
                        "restart.00000025.dat"]
    tecs = sorted(os.listdir(tmp_path / "TEC"))
    assert len(tecs) == 4 and host.tecplot_filename(s.maxima()["ctime"]) == tecs[-1]
    assert [host.tecplot_filename(k * dt)[:14] for k in (1, 11, 21, 25)] == [n[:14] for n in tecs]
    Qe, it, ct = host.restart_read(tmp_path / "restart.00000025.dat", t.N, m.ncell)
    assert it == 25 and np.array_equal(Qe, s.state()["Q"]) and ct == s.maxima()["ctime"]
    s.close()


def test_output_errors(tmp_path):
    m, t, ph, Q = ALL_SMALL["channel_n3"]()
    s = Solver(t, ph, precision="fp64")
    s.set_state(Q)
    with pytest.raises(SddcError):
        s.write_tecplot(tmp_path / "no_mesh.plt")  # no plot mesh yet
    s.write_restart(tmp_path / "missing_dir" / "r.dat", 1)
    with pytest.raises(SddcError) as e:
        s.output_wait()
    assert e.value.code == EIO
    s.output_wait()  # the failure is reported once
    s.write_restart(tmp_path / "ok.dat", 2)
    s.output_wait()
    assert (tmp_path / "ok.dat").exists()
    s.close()
