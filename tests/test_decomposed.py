"""Decomposed runs on the CPU: the oracle's restatement of the reference's
processor faces (PROCINTFLUX procintflux_all.f90:1-155, CYCREMFLUX
cycremflux_all.f90:1-155) and the rank exchange of sddc_b200.decomposed.

* One rank with no processor face runs the staged interface bit for bit as
  orc_rk_s5p3 (the staged RK_S5P3 and the split residual are the same code).
* Two and three ranks in one process, exchanging in lockstep, reproduce the
  single-domain oracle bit for bit on bilinear meshes: a cut face is
  evaluated on each side with that side's cell as the left cell, as the
  reference does, and the Rusanov flux is exactly antisymmetric under that
  swap (the unit normal and the state difference change sign exactly; sums
  commute), while both cells of a straight shared edge have the same face
  metrics.  On curved 8-node cells the two cells' metrics of a shared edge
  can differ in the last bit, and the runs agree to rounding.
* Two gloo ranks in two processes (world size 2), exchanging with
  torch.distributed point-to-point calls and a MAX all-reduce, give the same
  states bit for bit as the lockstep run.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import sddc_oracle as O
from helpers import case_cylinder, case_cylinder_curved, case_periodic, rel_l2
from sddc_b200 import decomposed, partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _route(parts, sbufs):
    """The receive buffer of every rank from every rank's send buffer."""
    rbufs = []
    for p in parts:
        rb = np.zeros_like(sbufs[p.rank])
        for peer, first, n in p.peers:
            back = [e for e in parts[peer].peers if e[0] == p.rank]
            assert len(back) == 1 and back[0][2] == n
            rb[first:first + n] = sbufs[peer][back[0][1]:back[0][1] + n]
        rbufs.append(rb)
    return rbufs


def lockstep(parts, physics, Q0, dt, nsteps, ncellglob):
    """Every rank's oracle in one process, stage by stage: pack, route,
    unpack, the residual up to the allreduce, MAX over ranks, the rest."""
    orcs = []
    for p in parts:
        o = O.Oracle(p.tables, physics, ncellglob=ncellglob)
        o.set_proc_faces(p.ibfproc)
        o.set_state(partition.scatter_state(Q0, p))
        orcs.append(o)
    for _ in range(nsteps):
        for stage in range(1, 6):
            for o in orcs:
                o.rk_begin_stage(stage)
            rb = _route(parts, [o.proc_pack() for o in orcs])
            for o, r in zip(orcs, rb):
                o.proc_unpack(r)
                o.compresid_local()
            mx = [o.local_maxima() for o in orcs]
            e, u = max(m[0] for m in mx), max(m[1] for m in mx)
            for o in orcs:
                o.set_global_maxima(e, u)
                o.compresid_finish()
                o.rk_end_stage(stage, dt)
    Q = partition.gather_state(parts, [o.state()["Q"] for o in orcs], Q0.shape[-1])
    return Q, orcs


CASES = {"cylinder": lambda: case_cylinder(nr=6, nt=12, N=4), "periodic": lambda: case_periodic(n=5, N=3)}
CURVED = {"cylinder_curved": lambda: case_cylinder_curved(nr=6, nt=12, N=4)}


@pytest.mark.parametrize("name", sorted(CASES))
def test_one_rank_staged_equals_rk_s5p3(name):
    m, t, ph, Q = CASES[name]()
    parts = partition.partition_tables(t, np.zeros(t.ncell, dtype=np.int32))
    assert parts[0].nproc == 0
    Qd, _ = lockstep(parts, ph, Q, 2e-3, 3, t.ncell)
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.rk_s5p3(2e-3, 3)
    assert np.array_equal(Qd, o.state()["Q"])


@pytest.mark.parametrize("name", sorted(CASES) + sorted(CURVED))
@pytest.mark.parametrize("nranks,scatter", [(2, False), (3, False), (3, True)])
def test_decomposed_matches_single_domain(name, nranks, scatter):
    m, t, ph, Q = {**CASES, **CURVED}[name]()
    if scatter:  # a part vector that is not a set of ranges
        part = np.random.default_rng(5).integers(0, nranks, t.ncell).astype(np.int32)
        part[:nranks] = np.arange(nranks)
    else:
        part = partition.split_cells(t.ncell, nranks)
    parts = partition.partition_tables(t, part)
    assert sum(p.tables.ncell for p in parts) == t.ncell
    assert all(p.nproc > 0 for p in parts)
    # every cut face is listed once on each side, in the same slot order
    for p in parts:
        for peer, first, n in p.peers:
            assert [e[2] for e in parts[peer].peers if e[0] == p.rank] == [n]
    Qd, orcs = lockstep(parts, ph, Q, 2e-3, 3, t.ncell)
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.rk_s5p3(2e-3, 3)
    ref = o.state()["Q"]
    if name in CASES:
        assert np.array_equal(Qd, ref)
        assert max(oo.maxima()["eigvmax"] for oo in orcs) == o.maxima()["eigvmax"]
    else:
        assert rel_l2(Qd, ref) <= 1e-15


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, name, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import datetime

    import sddc_oracle as O2
    from helpers import case_cylinder as cc, case_periodic as cp
    from sddc_b200 import decomposed as dec, partition as pt

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m, t, ph, Q = (cc(nr=6, nt=12, N=4) if name == "cylinder" else cp(n=5, N=3))
        parts = pt.partition_tables(t, pt.split_cells(t.ncell, world))
        p = parts[rank]
        o = O2.Oracle(p.tables, ph, ncellglob=t.ncell)
        o.set_proc_faces(p.ibfproc)
        o.set_state(pt.scatter_state(Q, p))
        rbuf = torch.zeros((p.nproc, t.N, 9), dtype=torch.float64)
        mx = torch.zeros(2, dtype=torch.float64)
        for _ in range(3):
            for stage in range(1, 6):
                o.rk_begin_stage(stage)
                sbuf = torch.from_numpy(o.proc_pack())
                dec.exchange_traces(dist, p, sbuf, rbuf)
                o.proc_unpack(rbuf.numpy())
                o.compresid_local()
                mx[:] = torch.tensor(o.local_maxima(), dtype=torch.float64)
                dec.allreduce_max(dist, mx)
                o.set_global_maxima(float(mx[0]), float(mx[1]))
                o.compresid_finish()
                o.rk_end_stage(stage, 2e-3)
        out[rank] = o.state()["Q"].tobytes(order="F")
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(CASES))
def test_gloo_world2_equals_lockstep(name):
    world = 2
    m, t, ph, Q = CASES[name]()
    parts = partition.partition_tables(t, partition.split_cells(t.ncell, world))
    Qd, _ = lockstep(parts, ph, Q, 2e-3, 3, t.ncell)
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_gloo_rank, args=(world, _free_port(), name, out), nprocs=world, start_method="spawn")
        got = [np.frombuffer(out[r], dtype=np.float64).reshape((9, t.N, t.N, parts[r].tables.ncell), order="F")
               for r in range(world)]
    assert np.array_equal(partition.gather_state(parts, got, t.ncell), Qd)
