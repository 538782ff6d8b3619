"""Partitioned meshes: one mesh split into parts that step together.

The reference runs one partition per MPI rank (src/main.F90:47-103): METIS
splits the mesh in a separate preprocessor (preProc_file/f23.f90), each rank
holds its cells plus one layer of partition ghosts, the conserved state of
those ghosts is exchanged after every RK stage (src/sr_mpiexchangecn.F90:1-96,
called from src/sr_RK.F90) and the time step is an MPI_Allreduce(MIN)
(src/main.F90:552).

Here a part is an ordinary mesh:

* its own cells (ascending global id, so local element 1 of the part that owns
  global element 1 is that element);
* the first halo layer: the other parts' cells that share a face with an own
  cell, iblank HP_IBLANK_HALO1 -- gradients and limiter are evaluated there
  exactly as the owner evaluates them, but no RK update;
* the second halo layer: the cells that share a face with the first,
  iblank HP_IBLANK_HALO2 (frozen), whose primitives feed the first layer's
  gradients, the face stencils of the viscous fluxes and the JST sweep;
* the boundary ghosts of those cells, plus ghosts of type HALO_EDGE_TYPE that
  close the second layer's outer faces (they only feed second-layer values
  that no own cell reads);
* the mesh's bounding-box nodes, appended unreferenced, so the far-field
  distances of src/sr_geometry.F90:295-347 come from the whole mesh's box.

Every own cell then reads, at every step, the inputs it reads in the whole
mesh, so the parts reproduce the single-mesh run bit for bit (one exception:
the stale flux of a face where HLLC takes no wave branch, a NaN state, comes
from the previous face of the part instead of the whole mesh).  Parts are
contiguous runs of the cells in Hilbert order of their centroids (METIS is not
available here).

Two ways to run them:

* PartitionedCase: all parts on one device as the cases of one batch
  (hp_set_halo copies each halo cell from its owner after every stage; the
  parts share one dt);
* RankPart: one part per process (several GPUs), with the exchange and the dt
  minimum done by a communicator through hp_set_exchange; DistComm is the
  torch.distributed one (NCCL between GPUs), ThreadComm runs several parts in
  one process (one host thread and one stream per part, copies ordered by
  CUDA events).
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass

import numpy as np

from . import cases
from ._lib import HP_EXCHANGE_FN, HP_IBLANK_HALO1, HP_IBLANK_HALO2, HP_X_DT, HpParams, lib
from .engine import Batch, Case, MeshArrays, _check, _ip

HALO_EDGE_TYPE = 2     # boundary type of the ghosts closing the second halo layer


def hilbert_keys(p: np.ndarray, bits: int = 10) -> np.ndarray:
    """Hilbert-curve index of each point (rows of p) on a 2^bits grid over
    the bounding cube (Skilling's transpose algorithm, vectorised)."""
    lo = p.min(axis=0)
    ext = max(float((p.max(axis=0) - lo).max()), 1e-300)
    top = (1 << bits) - 1
    q = np.clip(((p - lo) / ext * top).astype(np.int64), 0, top)
    X = [q[:, 0].copy(), q[:, 1].copy(), q[:, 2].copy()]
    Q = 1 << (bits - 1)
    while Q > 1:
        P = Q - 1
        for i in range(3):
            m = (X[i] & Q) != 0
            X[0] = np.where(m, X[0] ^ P, X[0])
            if i:
                t = np.where(m, 0, (X[0] ^ X[i]) & P)
                X[0] ^= t
                X[i] ^= t
        Q >>= 1
    X[1] ^= X[0]
    X[2] ^= X[1]
    t = np.zeros_like(X[0])
    Q = 1 << (bits - 1)
    while Q > 1:
        t = np.where((X[2] & Q) != 0, t ^ (Q - 1), t)
        Q >>= 1
    key = np.zeros_like(X[0])
    for i in range(3):
        X[i] ^= t
    for b in range(bits):
        for i in range(3):
            key |= ((X[i] >> b) & 1) << (3 * b + 2 - i)
    return key


@dataclass
class Part:
    spec: cases.CaseSpec      # the part as a case (own cells, halo 1, halo 2)
    own: np.ndarray           # global element ids (1-based) of local elements 1..nown
    halo: np.ndarray          # global ids of local elements nown+1.. (layer 1, then 2)
    nhalo1: int
    ghost_rows: np.ndarray    # per local ghost: row of the whole mesh's ghost list, -1 on halo edges

    @property
    def nown(self) -> int:
        return int(self.own.size)


@dataclass
class Partition:
    parts: list
    owner: np.ndarray         # [neles] part of each element
    local: np.ndarray         # [neles] local id (1-based) of each element in its owner part
    neles: int
    nghosts: int

    def halo_table(self):
        """(dst_case, dst_elem, src_case, src_elem) of hp_set_halo: every
        halo element of every part, from its owner."""
        dc, de, sc, se = [], [], [], []
        for p, part in enumerate(self.parts):
            g = part.halo
            dc.append(np.full(g.size, p, np.int32))
            de.append(np.arange(part.nown + 1, part.nown + 1 + g.size, dtype=np.int32))
            sc.append(self.owner[g - 1].astype(np.int32))
            se.append(self.local[g - 1].astype(np.int32))
        cat = lambda a: np.concatenate(a) if a else np.zeros(0, np.int32)  # noqa: E731
        return cat(dc), cat(de), cat(sc), cat(se)

    def exchange_lists(self, p: int):
        """Exchange of part p with its peers, in the order of the halo
        buffers: returns (peers, send_elem, send_counts, recv_elem,
        recv_counts), elements local to p (1-based).  Part p receives, from
        each peer q in ascending order, its halo cells owned by q in local
        order; it sends to q the own cells that q receives from p, in q's
        order."""
        part = self.parts[p]
        nown = part.nown
        src = self.owner[part.halo - 1]
        peers = sorted(set(int(q) for q in src) | {q for q, other in enumerate(self.parts)
                                                    if q != p and np.any(self.owner[other.halo - 1] == p)})
        send, scount, recv, rcount = [], [], [], []
        for q in peers:
            mine = np.flatnonzero(src == q)
            recv.append(nown + 1 + mine)
            rcount.append(mine.size)
            other = self.parts[q]
            theirs = other.halo[self.owner[other.halo - 1] == p]      # q's order
            send.append(self.local[theirs - 1])
            scount.append(theirs.size)
        cat = lambda a: np.concatenate(a).astype(np.int32) if a else np.zeros(0, np.int32)  # noqa: E731
        return peers, cat(send), np.array(scount, np.int64), cat(recv), np.array(rcount, np.int64)

    def scatter_state(self, cu: np.ndarray, ghost_prims: np.ndarray):
        """Per-part (cu, ghost prims) of a whole-mesh state; halo-edge ghosts
        take their parent's primitives from the part's own spec."""
        out = []
        for part in self.parts:
            loc = np.concatenate([part.own, part.halo]) - 1
            gp = part.spec.ghost_prims.copy()
            rows = part.ghost_rows
            gp[:, rows >= 0] = ghost_prims[:, rows[rows >= 0]]
            out.append((np.ascontiguousarray(cu[:, loc]), gp))
        return out

    def gather_state(self, states):
        """Whole-mesh (cu, ghost prims) from per-part (cu, ghost prims): each
        element and each ghost from the part that owns it (the ghost's parent)."""
        cu = np.zeros((10, self.neles))
        gp = np.zeros((6, self.nghosts))
        for part, (cp, gpp) in zip(self.parts, states):
            cu[:, part.own - 1] = cp[:, :part.nown]
            rows = part.ghost_rows
            keep = rows >= 0
            par = part.spec.mesh.ghost[:, 0]
            keep &= par <= part.nown
            gp[:, rows[keep]] = gpp[:, keep]
        return cu, gp


def partition_case(spec: cases.CaseSpec, nparts: int) -> Partition:
    """Split a case into nparts parts with two halo layers (module doc)."""
    m = spec.mesh
    ne, ng = m.neles, m.nghosts
    if nparts < 1 or nparts > ne:
        raise ValueError("nparts must be in [1, neles]")
    el = np.asarray(m.elem, np.int64)
    gh = np.asarray(m.ghost, np.int64)
    if ng and gh[:, 1].min() <= ne:
        raise ValueError("ghost ids alias element ids: not partitionable")
    nod = el[:, 0:4]
    xyz = np.stack([m.x, m.y, m.z], axis=1)
    xc = 0.25 * (xyz[nod[:, 0] - 1] + xyz[nod[:, 1] - 1] + xyz[nod[:, 2] - 1] + xyz[nod[:, 3] - 1])
    order = np.argsort(hilbert_keys(xc), kind="stable")
    owner = np.empty(ne, np.int64)
    owner[order] = (np.arange(ne) * nparts) // ne
    local = np.zeros(ne, np.int64)
    nb = el[:, 4:8]
    is_elem = nb <= ne
    grow = np.full(ne + ng + 2, -1, np.int64)            # ghost id -> ghost row
    grow[gh[:, 1]] = np.arange(ng)
    box_nodes = np.unique(np.concatenate([np.argmin(xyz, axis=0), np.argmax(xyz, axis=0)])) + 1
    parts_own = [np.flatnonzero(owner == p) + 1 for p in range(nparts)]
    for p, own in enumerate(parts_own):
        local[own - 1] = np.arange(1, own.size + 1)
    parts = []
    for p, own in enumerate(parts_own):
        inset = np.zeros(ne + 1, bool)
        inset[own] = True
        n1 = nb[own - 1][is_elem[own - 1]]
        h1 = np.unique(n1[~inset[n1]])
        inset[h1] = True
        n2 = nb[h1 - 1][is_elem[h1 - 1]]
        h2 = np.unique(n2[~inset[n2]])
        inset[h2] = True
        loc = np.concatenate([own, h1, h2])
        nloc = loc.size
        g2l = np.zeros(ne + 1, np.int64)
        g2l[loc] = np.arange(1, nloc + 1)
        # boundary ghosts of local cells (whole-mesh ghost order), then the
        # ghosts closing the second layer (cell order, face order)
        rows = np.flatnonzero(g2l[gh[:, 0]] > 0) if ng else np.zeros(0, np.int64)
        lnb = nb[loc - 1]
        lel = is_elem[loc - 1]
        edge = lel & (g2l[np.where(lel, lnb, 0)] == 0)
        ecell, eface = np.nonzero(edge)
        nrow, nedge = rows.size, ecell.size
        gid_of_row = np.full(ng + 1, 0, np.int64)
        gid_of_row[rows] = nloc + 1 + np.arange(nrow)
        lnc = np.where(lel, g2l[np.where(lel, lnb, 0)], gid_of_row[grow[np.where(lel, 0, lnb)]])
        lnc[ecell, eface] = nloc + 1 + nrow + np.arange(nedge)
        ghost = np.zeros((nrow + nedge, 4), np.int64)
        if nrow:
            ghost[:nrow, 0] = g2l[gh[rows, 0]]
            ghost[:nrow, 1] = gid_of_row[rows]
            ghost[:nrow, 2:4] = gh[rows, 2:4]
        ghost[nrow:, 0] = ecell + 1
        ghost[nrow:, 1] = nloc + 1 + nrow + np.arange(nedge)
        ghost[nrow:, 2] = HALO_EDGE_TYPE
        ghost[nrow:, 3] = eface + 1
        used = np.unique(np.concatenate([nod[loc - 1].ravel(), box_nodes]))
        n2l = np.zeros(m.nodes + 1, np.int64)
        n2l[used] = np.arange(1, used.size + 1)
        ib = el[loc - 1, 8].copy()
        k1 = slice(own.size, own.size + h1.size)
        k2 = slice(own.size + h1.size, nloc)
        ib[k1] = np.where(ib[k1] == 1, HP_IBLANK_HALO1, ib[k1])
        ib[k2] = np.where(ib[k2] == 1, HP_IBLANK_HALO2, ib[k2])
        elem = np.concatenate([n2l[nod[loc - 1]], lnc, ib[:, None]], axis=1).astype(np.int32)
        pm = MeshArrays(m.x[used - 1].copy(), m.y[used - 1].copy(), m.z[used - 1].copy(), elem,
                        ghost.astype(np.int32))
        cu = np.ascontiguousarray(spec.cu[:, loc - 1])
        fl = spec.flow
        gp = cases.ghost_prims_from_parents(pm, cu, fl["gamag"], fl["gamap"], fl["pinf"])
        if nrow:
            gp[:, :nrow] = spec.ghost_prims[:, rows]
        ps = cases.CaseSpec(f"{spec.name}.part{p}", pm, dict(fl), cu, gp, spec.steps, dict(spec.extra))
        grows = np.concatenate([rows, np.full(nedge, -1, np.int64)])
        parts.append(Part(ps, own, np.concatenate([h1, h2]), int(h1.size), grows))
    return Partition(parts, owner, local, ne, ng)


def _combine(diags, partition: Partition):
    """Whole-mesh diagnostics from per-part ones: time and dt are common, the
    residual maxima are the maxima over parts, NaN cells add up, |u_g| of
    element 1 comes from the part that owns it."""
    p1 = int(partition.owner[0])
    return {"time": diags[0]["time"], "dt": diags[0]["dt"], "velmag": diags[p1]["velmag"],
            "diff": np.max(np.stack([d["diff"] for d in diags]), axis=0),
            "nan_cells": np.sum(np.stack([d["nan_cells"] for d in diags]), axis=0)}


class PartitionedCase:
    """All parts of a partition on one device, as the cases of one batch
    coupled by hp_set_halo; the Case interface for the whole mesh."""

    def __init__(self, partition: Partition, params: HpParams):
        self.partition = partition
        self.batch = Batch([p.spec.mesh for p in partition.parts], params)
        dc, de, sc, se = (np.ascontiguousarray(a, np.int32) for a in partition.halo_table())
        _check(lib().hp_set_halo(self.batch.h, int(dc.size), _ip(dc), _ip(de), _ip(sc), _ip(se)), self.batch.h)

    def close(self):
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, time: float, cu: np.ndarray, ghost_prims: np.ndarray):
        for c, (cp, gp) in enumerate(self.partition.scatter_state(cu, ghost_prims)):
            self.batch.set_state(c, time, cp, gp)

    def step(self, nsteps: int, diagnostics: bool = True):
        d = self.batch.step(nsteps, diagnostics)
        return None if d is None else _combine(d, self.partition)

    def step_timed(self, nsteps: int) -> float:
        return self.batch.step_timed(nsteps)

    def state(self):
        st = [self.batch.state(c) for c in range(self.batch.ncase)]
        cu, gp = self.partition.gather_state([(s[1], s[2]) for s in st])
        return st[0][0], cu, gp


# --- one part per process ------------------------------------------------------

class RankPart:
    """Part `rank` of a partition in a single-case handle, exchanging with the
    other parts through `comm` at the library's exchange points:

    * HP_X_DT: comm.min_i64(dtmin, stream) -- the part's partial dt minimum
      (a device int64 view of hp_dtmin_ptr) becomes the minimum over parts;
    * HP_X_HALO: hp_halo_pack into the send buffer, comm.exchange of the
      per-peer blocks, hp_halo_unpack from the receive buffer.

    comm is DistComm (torch.distributed, one GPU per process) or ThreadComm
    (parts of one process).  Buffers are torch CUDA tensors."""

    def __init__(self, partition: Partition, rank: int, params: HpParams, comm):
        import torch
        self.partition, self.rank, self.comm = partition, rank, comm
        part = partition.parts[rank]
        self.case = Case(part.spec.mesh, params)
        peers, send, scount, recv, rcount = partition.exchange_lists(rank)
        self.peers, self.scount, self.rcount = peers, scount, rcount
        L = lib()
        _check(L.hp_set_halo_lists(self.case.h, int(send.size), _ip(send), int(recv.size), _ip(recv)), self.case.h)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.sendbuf = torch.empty(10 * max(send.size, 1), dtype=torch.float64, device=dev)
        self.recvbuf = torch.empty(10 * max(recv.size, 1), dtype=torch.float64, device=dev)
        ptr = ctypes.POINTER(ctypes.c_uint64)()
        _check(L.hp_dtmin_ptr(self.case.h, ctypes.byref(ptr)), self.case.h)
        self.dtmin = torch.as_tensor(_DeviceWord(ctypes.cast(ptr, ctypes.c_void_p).value), device=dev)
        self._fn = HP_EXCHANGE_FN(self._exchange)
        self.error = None
        _check(L.hp_set_exchange(self.case.h, self._fn, None), self.case.h)

    def _exchange(self, _user, point, stream):
        try:
            if point == HP_X_DT:
                self.comm.min_i64(self.dtmin, stream)
            else:
                L = lib()
                L.hp_halo_pack(self.case.h, ctypes.c_void_p(self.sendbuf.data_ptr()))
                self.comm.exchange(self.sendbuf, self.scount, self.recvbuf, self.rcount, self.peers, stream)
                L.hp_halo_unpack(self.case.h, ctypes.c_void_p(self.recvbuf.data_ptr()))
        except Exception as e:        # raised back to the caller after the step
            if self.error is None:
                self.error = e

    def set_state(self, time: float, cu_part: np.ndarray, ghost_prims_part: np.ndarray):
        self.case.set_state(time, cu_part, ghost_prims_part)

    def step(self, nsteps: int, diagnostics: bool = True):
        d = self.case.step(nsteps, diagnostics)
        if self.error is not None:
            raise self.error
        return d

    def state(self):
        return self.case.state()

    def close(self):
        lib().hp_set_exchange(self.case.h, HP_EXCHANGE_FN(), None)     # NULL: no callback
        self.case.close()


class _DeviceWord:
    """One int64 of device memory, for torch.as_tensor."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<i8", "data": (ptr, False), "version": 3}


class DistComm:
    """torch.distributed on the library's stream: one part per rank (NCCL
    between GPUs).  With stream None the same calls run on CPU tensors, as
    the gloo tests do."""

    def __init__(self, group=None):
        self.group = group

    def _on(self, stream):
        import contextlib

        import torch
        if stream is None:
            return contextlib.nullcontext()
        return torch.cuda.stream(torch.cuda.ExternalStream(stream))

    def min_i64(self, t, stream):
        import torch.distributed as dist
        with self._on(stream):
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)

    def exchange(self, sendbuf, scount, recvbuf, rcount, peers, stream):
        import torch.distributed as dist
        ops, so, ro = [], 0, 0
        for q, ns, nr in zip(peers, scount, rcount):
            ns, nr = int(ns), int(nr)
            if ns:
                ops.append(dist.P2POp(dist.isend, sendbuf[10 * so:10 * (so + ns)], q, self.group))
            if nr:
                ops.append(dist.P2POp(dist.irecv, recvbuf[10 * ro:10 * (ro + nr)], q, self.group))
            so += ns
            ro += nr
        with self._on(stream):
            for w in (dist.batch_isend_irecv(ops) if ops else []):
                w.wait()


class ThreadComm:
    """Several parts in one process: one host thread and one CUDA stream per
    part.  Every exchange runs in three phases separated by barriers: each
    part posts its buffer and an event; each part waits for its peers'
    events on its own stream, copies its blocks out of their buffers and
    posts a second event; each part's stream waits for the second events of
    the peers that read its buffer, before the buffer is written again.  The
    ordering is host barriers plus CUDA events; no kernel waits on another.
    A barrier that times out breaks, so a failed part ends the others'
    steps with an error instead of a hang."""

    def __init__(self, nparts: int, timeout: float = 120.0):
        self.n = nparts
        self.barrier = threading.Barrier(nparts, timeout=timeout)
        self.ready = [None] * nparts      # (tensor, event, block offsets by peer)
        self.read = [None] * nparts       # event after this part's reads of the others

    def bind(self, rank: int):
        return _ThreadRank(self, rank)


class _ThreadRank:
    def __init__(self, hub: ThreadComm, rank: int):
        self.hub, self.rank = hub, rank

    def _post(self, s, buf, offs):
        import torch
        ev = torch.cuda.Event()
        ev.record(s)
        self.hub.ready[self.rank] = (buf, ev, offs)
        self.hub.barrier.wait()

    def _finish(self, s, readers):
        import torch
        hub = self.hub
        ev = torch.cuda.Event()
        ev.record(s)
        hub.read[self.rank] = ev
        hub.barrier.wait()
        for q in readers:
            s.wait_event(hub.read[q])

    def min_i64(self, t, stream):
        import torch
        hub = self.hub
        s = torch.cuda.ExternalStream(stream)
        with torch.cuda.stream(s):
            self._post(s, t, None)
            try:
                for q in range(hub.n):
                    s.wait_event(hub.ready[q][1])
                m = torch.min(torch.cat([hub.ready[q][0] for q in range(hub.n)])).reshape(1)
            except BaseException:
                hub.barrier.abort()      # the peers fail at once, not at the timeout
                raise
            self._finish(s, [q for q in range(hub.n) if q != self.rank])
            t.copy_(m)

    def exchange(self, sendbuf, scount, recvbuf, rcount, peers, stream):
        import torch
        hub, r = self.hub, self.rank
        s = torch.cuda.ExternalStream(stream)
        offs, o = {}, 0
        for q, ns in zip(peers, scount):
            offs[q] = (o, int(ns))
            o += int(ns)
        with torch.cuda.stream(s):
            self._post(s, sendbuf, offs)
            try:
                ro = 0
                for q, nr in zip(peers, rcount):
                    nr = int(nr)
                    buf, qev, qoffs = hub.ready[q]
                    so, ns = qoffs.get(r, (0, 0))
                    if ns != nr:
                        raise RuntimeError(f"part {r} expects {nr} cells from part {q}, which sends {ns}")
                    if nr:
                        s.wait_event(qev)
                        recvbuf[10 * ro:10 * (ro + nr)].copy_(buf[10 * so:10 * (so + ns)])
                    ro += nr
            except BaseException:
                # a part that fails between posting and finishing would leave
                # its peers at the second barrier until the timeout; breaking
                # the barrier ends their exchange at once with an error
                hub.barrier.abort()
                raise
            self._finish(s, peers)
