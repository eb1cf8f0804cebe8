"""Decomposed runs: one partition of a case per rank, one GPU per rank.

The exchange each stage needs is the one of the reference's MPI ranks
(procintflux_all.f90:28-80, cycremflux_all.f90:28-80, compflux.f90:10-11):
every processor face's N x 9 trace of its own cell goes to the rank on the
other side, and both running maxima are reduced with MAX.  With
``partition.Part`` ordering the processor faces by peer and then by global
face, the traffic with one peer is one contiguous slot range each way, sent
and received with torch.distributed point-to-point calls (NCCL between GPUs;
gloo between CPU ranks), so the remote traces land in this rank's own
buffer before any kernel reads them.

``DecomposedSolver`` runs one rank's partition on this process's GPU: the
drop-in context holds the processor faces (``sddc_set_proc_faces``), packs
the traces of every stage into a send buffer and, between stages, calls
back into the host (``sddc_set_exchange``), which exchanges them and the
maxima on the context's stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .partition import Part


def exchange_traces(dist, part: Part, sbuf, rbuf, group=None) -> None:
    """Send each peer's slot range of sbuf and receive the same range of
    rbuf from it (tensors shaped (nproc, ...), slot-major)."""
    ops = []
    for peer, first, n in part.peers:
        ops.append(dist.P2POp(dist.isend, sbuf[first:first + n], peer, group))
        ops.append(dist.P2POp(dist.irecv, rbuf[first:first + n], peer, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


def allreduce_max(dist, t, group=None) -> None:
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)


class DecomposedSolver:
    """One rank of a decomposed case on the current GPU (torch.distributed
    must be initialised with the NCCL backend; one process per GPU)."""

    def __init__(self, part: Part, physics, dist, precision="fp64", ncellglob: int | None = None,
                 cells_per_cta: int = 0, group=None):
        import torch

        from .solver import Solver

        self.part, self.dist, self.group = part, dist, group
        self.solver = Solver(part.tables, physics, precision=precision, cells_per_cta=cells_per_cta,
                             ncellglob=ncellglob, proc_faces=part.ibfproc)
        elem = torch.float32 if self.solver.precision == 2 else torch.float64
        dev = torch.device("cuda", torch.cuda.current_device())
        n = max(part.nproc, 1)
        self.sbuf = torch.zeros((n, part.tables.N, 9), dtype=elem, device=dev)
        self.rbuf = torch.zeros_like(self.sbuf)
        self.maxima = torch.zeros(2, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(self.solver.stream_handle())
        self._torch = torch

        def exchange(user):
            with torch.cuda.stream(self.stream):
                exchange_traces(dist, part, self.sbuf[:part.nproc], self.rbuf[:part.nproc], group)
                allreduce_max(dist, self.maxima, group)
            return 0

        self.solver.set_exchange(exchange, self.sbuf.data_ptr(), self.rbuf.data_ptr(), self.maxima.data_ptr())

    def set_state(self, Q_local, **kw):
        self.solver.set_state(Q_local, **kw)

    def rk_s5p3(self, dt, nsteps=1):
        self.solver.rk_s5p3(dt, nsteps)

    def state(self):
        return self.solver.state()

    def close(self):
        self.solver.close()


def trace_dtype(precision) -> type:
    """numpy type of the exchanged traces of a form (float32 for the mixed
    form, whose traces are FP32)."""
    return np.float32 if precision in ("mixed", 2) else np.float64
