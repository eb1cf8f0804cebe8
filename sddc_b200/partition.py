"""Domain decomposition of a case over ranks (the reference's MPI partitions).

The reference reads a METIS cell partition (READ_METIS,
readGRIDinfo.f90:119-153), gives each rank the faces of its cells and turns a
face whose other cell lives on another rank into a processor face (IBFPROC;
a periodic pair split over two ranks is a remote cyclic face, IBFCYCREM,
connect_bdry.f90:255-314).  In every residual each rank sends, per
processor face, the N x 9 trace of its own cell at the face's flux points
(procintflux_all.f90:28-99, cycremflux_all.f90:28-80) and evaluates the face
with its own cell as the left cell; both running maxima are reduced with
MPI_ALLREDUCE(MAX) (compflux.f90:10-11).

Here the partition works on the set-up tables of the whole case
(``host.build_tables``): ``partition_tables`` cuts them into one ``Part`` per
rank with local cell and face numbers.  A processor face keeps the reference's
convention IF2C(K,1) = own cell, IF2C(K,3) = its local face.  The processor
faces of a rank are ordered by peer rank, then by the global face (interior
face id, or periodic pair id), so that both sides of every cut list their
shared faces in the same order: the exchange with one peer is one contiguous
slot range in each direction (``Part.peers``).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .host import Tables


@dataclasses.dataclass
class Part:
    rank: int
    cells: np.ndarray    # global cell ids (0-based) of this rank, ascending; local cell i is cells[i]
    tables: Tables       # local tables (cells and faces renumbered)
    ibfproc: np.ndarray  # local face ids (1-based) of the processor faces, in slot order
    proc_peer: np.ndarray  # rank on the other side of each processor face
    peers: list          # [(peer, first slot, slots)] in peer order

    @property
    def nproc(self) -> int:
        return int(self.ibfproc.shape[0])


def split_cells(ncell: int, nranks: int) -> np.ndarray:
    """A part vector of contiguous cell-id ranges of nearly equal size (the
    role of the METIS partition file)."""
    bounds = np.linspace(0, ncell, nranks + 1).round().astype(int)
    part = np.empty(ncell, dtype=np.int32)
    for r in range(nranks):
        part[bounds[r]:bounds[r + 1]] = r
    return part


def partition_tables(t: Tables, part: np.ndarray) -> list[Part]:
    """One Part per rank of the part vector (rank of each global cell)."""
    part = np.asarray(part, dtype=np.int64)
    if part.shape != (t.ncell,):
        raise ValueError("part must give a rank for every cell")
    nranks = int(part.max()) + 1
    IF2C = np.asarray(t.IF2C)
    out = []
    for r in range(nranks):
        cells = np.flatnonzero(part == r)
        if cells.size == 0:
            raise ValueError(f"rank {r} owns no cell")
        g2l = np.full(t.ncell, -1, dtype=np.int64)
        g2l[cells] = np.arange(cells.size)
        faces = []   # local face rows [IF2C(4)], IF2V
        gface = {}   # global face id -> local face id (1-based)

        def add(row, gf):
            faces.append((row, t.IF2V[gf - 1]))
            gface[(gf, row[0])] = len(faces)
            return len(faces)

        inter, procs = [], []  # procs: (peer, key, local face)
        for f in np.asarray(t.ibfinter):
            cl, cr, lfl, lfr = (int(x) for x in IF2C[f - 1])
            il, ir = part[cl - 1] == r, part[cr - 1] == r
            if il and ir:
                inter.append(add([g2l[cl - 1] + 1, g2l[cr - 1] + 1, lfl, lfr], f))
            elif il:
                procs.append((int(part[cr - 1]), (0, int(f)), add([g2l[cl - 1] + 1, 0, lfl, 0], f)))
            elif ir:
                procs.append((int(part[cl - 1]), (0, int(f)), add([g2l[cr - 1] + 1, 0, lfr, 0], f)))
        bnd = {}
        for name in ("ibfinl", "ibfout", "ibfwal", "ibfsymp", "ibfree"):
            lst = []
            for f in np.asarray(getattr(t, name)):
                c, _, lf, _ = (int(x) for x in IF2C[f - 1])
                if part[c - 1] == r:
                    lst.append(add([g2l[c - 1] + 1, 0, lf, 0], f))
            bnd[name] = np.asarray(lst, dtype=np.int32)
        pairs = []
        cyc = np.asarray(t.cyc2fpair)
        for q in range(cyc.shape[0]):
            K1, K2 = int(cyc[q, 0]), int(cyc[q, 1])
            c1, c2 = int(IF2C[K1 - 1, 0]), int(IF2C[K2 - 1, 0])
            i1, i2 = part[c1 - 1] == r, part[c2 - 1] == r
            if i1 and i2:
                a = add([g2l[c1 - 1] + 1, 0, int(IF2C[K1 - 1, 2]), 0], K1)
                b = add([g2l[c2 - 1] + 1, 0, int(IF2C[K2 - 1, 2]), 0], K2)
                pairs.append((a, b))
            elif i1:
                procs.append((int(part[c2 - 1]), (1, q), add([g2l[c1 - 1] + 1, 0, int(IF2C[K1 - 1, 2]), 0], K1)))
            elif i2:
                procs.append((int(part[c1 - 1]), (1, q), add([g2l[c2 - 1] + 1, 0, int(IF2C[K2 - 1, 2]), 0], K2)))
        procs.sort(key=lambda x: (x[0], x[1]))
        nf = len(faces)
        lIF2C = np.zeros((nf, 4), np.int32, order="F")
        lIF2V = np.zeros((nf, 2), np.int32, order="F")
        for k, (row, v) in enumerate(faces):
            lIF2C[k] = row
            lIF2V[k] = v
        cyc_l = np.zeros((len(pairs), 2), np.int32, order="F")
        for k, (a, b) in enumerate(pairs):
            cyc_l[k] = (a, b)
        counts = dict(t.counts)
        counts.update(ncell=int(cells.size), nface=nf, ninter=len(inter), ninlet=len(bnd["ibfinl"]),
                      noutlet=len(bnd["ibfout"]), nwall=len(bnd["ibfwal"]), nsymp=len(bnd["ibfsymp"]),
                      nfree=len(bnd["ibfree"]), npair=len(pairs))
        lt = Tables(N=t.N, ncell=int(cells.size), Lmat=t.Lmat, Mmat=t.Mmat, Xs=t.Xs, Xf=t.Xf,
                    S1=np.asfortranarray(t.S1[..., cells]), S2=np.asfortranarray(t.S2[..., cells]),
                    Jac=np.asfortranarray(t.Jac[..., cells]), xxsolu=np.asfortranarray(t.xxsolu[..., cells]),
                    IF2C=lIF2C, IF2V=lIF2V, ibfinter=np.asarray(inter, dtype=np.int32),
                    ibfinl=bnd["ibfinl"], ibfout=bnd["ibfout"], ibfwal=bnd["ibfwal"], ibfsymp=bnd["ibfsymp"],
                    ibfree=bnd["ibfree"], cyc2fpair=cyc_l, ivcell=np.asfortranarray(t.ivcell[cells]),
                    counts=counts, dxcycl=t.dxcycl, dycycl=t.dycycl)
        ibfproc = np.asarray([p[2] for p in procs], dtype=np.int32)
        peer = np.asarray([p[0] for p in procs], dtype=np.int32)
        peers = []
        for p in sorted(set(peer.tolist())):
            idx = np.flatnonzero(peer == p)
            peers.append((p, int(idx[0]), int(idx.size)))
        out.append(Part(rank=r, cells=cells, tables=lt, ibfproc=ibfproc, proc_peer=peer, peers=peers))
    return out


def scatter_state(Q: np.ndarray, p: Part) -> np.ndarray:
    """This rank's slice (9,N,N,local cells) of a global state."""
    return np.asfortranarray(Q[..., p.cells])


def gather_state(parts: list[Part], locals_: list[np.ndarray], ncell: int) -> np.ndarray:
    """The global state from every rank's slice."""
    q0 = locals_[0]
    Q = np.zeros(q0.shape[:-1] + (ncell,), dtype=q0.dtype, order="F")
    for p, q in zip(parts, locals_):
        Q[..., p.cells] = q
    return Q
