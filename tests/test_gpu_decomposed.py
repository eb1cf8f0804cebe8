"""Decomposed runs of the drop-in on the GPU, through the C ABI
(sddc_set_proc_faces, sddc_set_exchange), against the CPU oracle.

Only one GPU is available to these tests, so two and three ranks run as
contexts on the same GPU, each driven by its own host thread.  Their
exchange is host-synchronised: a rank's callback waits for its stream, meets
the other threads at a barrier, copies the peers' send buffers into its
receive buffer and reduces the maxima on its own stream, and meets them
again before returning; no kernel ever waits for another context.  On
bilinear meshes the reference's processor-face evaluation reproduces the
single-domain bits (tests/test_decomposed.py), so the exact form of the
decomposed run equals the oracle's single-domain run bit for bit.

With one rank, sddc_b200.decomposed.DecomposedSolver exchanges through
torch.distributed's NCCL backend (an all-reduce of the maxima on the
context's stream) and equals the plain context bit for bit.
"""
import datetime
import os
import socket
import threading

import numpy as np
import pytest
import torch

import sddc_oracle as O
from helpers import case_cylinder, case_periodic, rel_l2
from sddc_b200 import decomposed, partition
from sddc_b200.solver import SddcError, Solver

pytestmark = pytest.mark.gpu

CASES = {"cylinder": lambda: case_cylinder(nr=6, nt=12, N=4), "periodic": lambda: case_periodic(n=5, N=5)}


class Ranks:
    """Contexts of every rank on this GPU, exchanging through the host."""

    def __init__(self, parts, physics, precision, ncellglob):
        self.parts = parts
        n = len(parts)
        self.bar = threading.Barrier(n, timeout=60)
        dt = torch.float32 if precision == "mixed" else torch.float64
        self.solvers, self.sbuf, self.rbuf, self.mx, self.tmp, self.streams = [], [], [], [], [], []
        for p in parts:
            s = Solver(p.tables, physics, precision=precision, ncellglob=ncellglob, proc_faces=p.ibfproc)
            sb = torch.zeros((max(p.nproc, 1), p.tables.N, 9), dtype=dt, device="cuda")
            self.solvers.append(s)
            self.sbuf.append(sb)
            self.rbuf.append(torch.zeros_like(sb))
            self.mx.append(torch.zeros(2, dtype=torch.float64, device="cuda"))
            self.tmp.append(torch.zeros(2, dtype=torch.float64, device="cuda"))
            self.streams.append(torch.cuda.ExternalStream(s.stream_handle()))
        for r, s in enumerate(self.solvers):
            s.set_exchange(self._callback(r), self.sbuf[r].data_ptr(), self.rbuf[r].data_ptr(),
                           self.mx[r].data_ptr())

    def _callback(self, r):
        def fn(user):
            st = self.streams[r]
            st.synchronize()
            self.bar.wait()
            with torch.cuda.stream(st):
                for peer, first, n in self.parts[r].peers:
                    (pfirst,) = [e[1] for e in self.parts[peer].peers if e[0] == r]
                    self.rbuf[r][first:first + n].copy_(self.sbuf[peer][pfirst:pfirst + n])
                m = self.mx[0].clone()
                for q in range(1, len(self.mx)):
                    m = torch.maximum(m, self.mx[q])
                self.tmp[r].copy_(m)
            st.synchronize()
            self.bar.wait()
            with torch.cuda.stream(st):
                self.mx[r].copy_(self.tmp[r])
            st.synchronize()
            self.bar.wait()
            return 0
        return fn

    def run(self, fn):
        """fn(rank, solver) on every rank, one host thread each."""
        errs = []

        def body(r):
            try:
                torch.cuda.set_device(0)
                fn(r, self.solvers[r])
            except BaseException as e:  # noqa: BLE001
                errs.append(e)
                self.bar.abort()

        th = [threading.Thread(target=body, args=(r,)) for r in range(len(self.solvers))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]

    def close(self):
        for s in self.solvers:
            s.close()


def _run(name, nranks, precision, nsteps=3, dt=2e-3):
    m, t, ph, Q = CASES[name]()
    parts = partition.partition_tables(t, partition.split_cells(t.ncell, nranks))
    rk = Ranks(parts, ph, precision, t.ncell)
    out = [None] * nranks

    def body(r, s):
        s.set_state(partition.scatter_state(Q, parts[r]))
        s.rk_s5p3(dt, nsteps)
        out[r] = s.state()["Q"]

    rk.run(body)
    rk.close()
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.rk_s5p3(dt, nsteps)
    return partition.gather_state(parts, out, t.ncell), o.state()["Q"], o


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("nranks", [2, 3])
def test_decomposed_exact_equals_oracle(name, nranks):
    got, ref, _ = _run(name, nranks, "fp64_exact")
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision,bar", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_decomposed_forms(name, precision, bar):
    got, ref, _ = _run(name, 2, precision, nsteps=1)
    assert rel_l2(got, ref) <= bar


def test_decomposed_residual_and_maxima():
    """sddc_compresid of a decomposed state: the residual and all nine
    gradients of every rank equal the single-domain oracle's, and every
    rank ends with the global running maxima."""
    m, t, ph, Q = CASES["cylinder"]()
    parts = partition.partition_tables(t, partition.split_cells(t.ncell, 2))
    rk = Ranks(parts, ph, "fp64_exact", t.ncell)
    res, mx = [None, None], [None, None]

    def body(r, s):
        s.set_state(partition.scatter_state(Q, parts[r]))
        s.compresid()
        s.compresid()
        g = s.state(resid=True, nablaQs=True)
        res[r] = (g["resid"], g["nablaQs"])
        mx[r] = s.maxima()

    rk.run(body)
    rk.close()
    o = O.Oracle(t, ph)
    o.set_state(Q)
    o.compresid()
    o.compresid()
    a = o.state()
    assert np.array_equal(partition.gather_state(parts, [x[0] for x in res], t.ncell), a["resid"])
    assert np.array_equal(partition.gather_state(parts, [x[1] for x in res], t.ncell), a["nablaQs"])
    for r in range(2):
        assert mx[r]["eigvmax"] == o.maxima()["eigvmax"] and mx[r]["umax"] == o.maxima()["umax"]


def test_processor_faces_need_an_exchange():
    m, t, ph, Q = CASES["cylinder"]()
    parts = partition.partition_tables(t, partition.split_cells(t.ncell, 2))
    s = Solver(parts[0].tables, ph, proc_faces=parts[0].ibfproc)
    s.set_state(partition.scatter_state(Q, parts[0]))
    with pytest.raises(SddcError, match="sddc_set_exchange"):
        s.rk_s5p3(1e-3, 1)
    s.close()
    # without the declaration the cut faces are in no list
    with pytest.raises(SddcError, match="processor face"):
        Solver(parts[0].tables, ph)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_decomposed_solver_nccl_world1():
    import torch.distributed as dist

    m, t, ph, Q = CASES["periodic"]()
    parts = partition.partition_tables(t, np.zeros(t.ncell, dtype=np.int32))
    store = dist.TCPStore("127.0.0.1", _free_port(), 1, True, timeout=datetime.timedelta(seconds=60))
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        d = decomposed.DecomposedSolver(parts[0], ph, dist, precision="fp64_exact")
        d.set_state(Q)
        d.rk_s5p3(2e-3, 3)
        got = d.state()["Q"]
        d.close()
    finally:
        dist.destroy_process_group()
    s = Solver(t, ph, precision="fp64_exact")
    s.set_state(Q)
    s.rk_s5p3(2e-3, 3)
    assert np.array_equal(got, s.state()["Q"])
    s.close()
