"""Partitioned meshes (hydraphase.partition; the reference's MPI partitions,
src/sr_mpiexchangecn.F90 and the dt allreduce of src/main.F90:552).

CPU: the parts' structure -- own cells partition the mesh; the first halo
layer is the face neighbours of the own cells, the second theirs; every
local element keeps its nodes, its whole-mesh neighbours and boundary
ghosts, and the second layer's open faces are closed by halo-edge ghosts;
the whole mesh's bounding box is kept; states scatter and gather exactly;
the per-peer exchange lists agree pairwise.  Two and three gloo ranks run
the exchange (the halo takes the owners' values) and the dt minimum through
DistComm, with the library's pack/unpack done in numpy.
GPU: the parts run as one coupled batch (hp_set_halo) and as one handle per
part exchanging through hp_set_exchange (ThreadComm: one host thread and
stream per part) reproduce the single-mesh FP64 parity run bit for bit
(state, ghosts, time, dt, residuals, |u_g| of cell 1), which itself equals
the oracle.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hydraphase import PREC_FP64_PARITY, PREC_MIXED, Case, cases
from hydraphase._lib import HP_IBLANK_HALO1, HP_IBLANK_HALO2
from hydraphase.partition import HALO_EDGE_TYPE, partition_case

SPECS = {
    "shock_bubble": lambda: cases.shock_bubble(n=6, alpha_min=0.1),
    "shock_bubble_ref": lambda: cases.shock_bubble(n=6, alpha_min=0.1, reference_scheme=True),
    "cylinder": lambda: cases.cylinder(nr=6, nt=16, nz=2),
}


def _neighbours(el, ids, ne):
    n = el[ids - 1, 4:8].ravel()
    return np.unique(n[n <= ne])


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("nparts", [1, 2, 5, 37])
def test_parts_structure(name, nparts):
    spec = SPECS[name]()
    m = spec.mesh
    el = m.elem.astype(np.int64)
    ne = m.neles
    P = partition_case(spec, nparts)
    own_all = np.concatenate([p.own for p in P.parts])
    np.testing.assert_array_equal(np.sort(own_all), np.arange(1, ne + 1))
    xyz = np.stack([m.x, m.y, m.z], 1)
    for p, part in enumerate(P.parts):
        pm = part.spec.mesh
        assert np.all(np.diff(part.own) > 0) and np.all(P.owner[part.own - 1] == p)
        np.testing.assert_array_equal(P.local[part.own - 1], np.arange(1, part.nown + 1))
        h1 = part.halo[:part.nhalo1]
        h2 = part.halo[part.nhalo1:]
        n1 = _neighbours(el, part.own, ne)
        np.testing.assert_array_equal(h1, np.setdiff1d(n1, part.own))
        n2 = _neighbours(el, h1, ne) if h1.size else np.zeros(0, np.int64)
        np.testing.assert_array_equal(h2, np.setdiff1d(n2, np.concatenate([part.own, h1])))
        loc = np.concatenate([part.own, part.halo])
        nloc = loc.size
        lel = pm.elem.astype(np.int64)
        ib = lel[:, 8]
        assert np.all(ib[:part.nown] == 1)
        assert np.all(ib[part.nown:part.nown + part.nhalo1] == HP_IBLANK_HALO1)
        assert np.all(ib[part.nown + part.nhalo1:] == HP_IBLANK_HALO2)
        lxyz = np.stack([pm.x, pm.y, pm.z], 1)
        np.testing.assert_array_equal(lxyz[lel[:, :4] - 1], xyz[el[loc - 1, :4] - 1])
        np.testing.assert_array_equal(lxyz.min(0), xyz.min(0))
        np.testing.assert_array_equal(lxyz.max(0), xyz.max(0))
        ng = pm.nghosts
        gh = pm.ghost.astype(np.int64)
        np.testing.assert_array_equal(gh[:, 1], nloc + 1 + np.arange(ng))
        np.testing.assert_array_equal(lel[gh[:, 0] - 1, 4 + gh[:, 3] - 1], gh[:, 1])
        gpos = {int(g): r for r, g in enumerate(m.ghost[:, 1])}
        for a in range(nloc):
            for k in range(4):
                gn, ln = el[loc[a] - 1, 4 + k], lel[a, 4 + k]
                if gn <= ne and ln <= nloc:
                    assert loc[ln - 1] == gn
                elif gn > ne:
                    r = part.ghost_rows[ln - nloc - 1]
                    assert r == gpos[int(gn)]
                else:          # a face of the second layer out of the part
                    assert a >= part.nown + part.nhalo1 and ln > nloc
                    assert gh[ln - nloc - 1, 2] == HALO_EDGE_TYPE and part.ghost_rows[ln - nloc - 1] == -1
    dc, de, sc, se = P.halo_table()
    for c, e, q, s in zip(dc, de, sc, se):
        part = P.parts[c]
        g = part.halo[e - part.nown - 1]
        assert P.owner[g - 1] == q and P.parts[q].own[s - 1] == g
    cu, gp = P.gather_state([(a, b) for a, b in P.scatter_state(spec.cu, spec.ghost_prims)])
    np.testing.assert_array_equal(cu, spec.cu)
    np.testing.assert_array_equal(gp, spec.ghost_prims)
    for p in range(nparts):
        peers, send, sc_, recv, rc_ = P.exchange_lists(p)
        for j, q in enumerate(peers):
            qp, qsend, qsc, qrecv, qrc = P.exchange_lists(q)
            i = qp.index(p)
            assert sc_[j] == qrc[i] and rc_[j] == qsc[i]
            mine = send[sc_[:j].sum():sc_[:j + 1].sum()]
            theirs = qrecv[qrc[:i].sum():qrc[:i + 1].sum()]
            qpart = P.parts[q]
            np.testing.assert_array_equal(P.parts[p].own[mine - 1], qpart.halo[theirs - qpart.nown - 1])


def test_partition_rejects_aliased_ghosts():
    spec = SPECS["shock_bubble"]()
    m = spec.mesh
    gh = m.ghost.copy()
    gh[0, 1] = 1
    spec.mesh = type(m)(m.x, m.y, m.z, m.elem, gh)
    with pytest.raises(ValueError):
        partition_case(spec, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from hydraphase.partition import DistComm
    spec = SPECS["cylinder"]()
    P = partition_case(spec, world)
    part = P.parts[rank]
    loc = np.concatenate([part.own, part.halo])
    new = spec.cu * 1.5 + np.arange(spec.mesh.neles)[None, :]      # the "stage update"
    cn = np.zeros((10, loc.size))
    cn[:, :part.nown] = new[:, part.own - 1]                         # halo still stale
    peers, send, scount, recv, rcount = P.exchange_lists(rank)
    sendbuf = torch.from_numpy(np.ascontiguousarray(cn[:, send - 1].T).reshape(-1))
    recvbuf = torch.zeros(10 * recv.size, dtype=torch.float64)
    comm = DistComm()
    comm.exchange(sendbuf, scount, recvbuf, rcount, peers, None)
    cn[:, recv - 1] = recvbuf.numpy().reshape(-1, 10).T
    ok = bool(np.array_equal(cn, new[:, loc - 1]))
    word = torch.tensor([1000 + 7 * rank], dtype=torch.int64)
    comm.min_i64(word, None)
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([ok, int(word[0])]))


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo(tmp_path, world):
    mp.spawn(_exchange_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        ok, word = np.load(tmp_path / f"r{r}.npy")
        assert ok and word == 1000


class _FakeEvent:
    def record(self, stream=None):
        pass


class _FakeStream:
    def __init__(self, handle=None):
        pass

    def wait_event(self, ev):
        pass


def test_thread_exchange_failure_ends_all_parts_promptly(monkeypatch):
    """A part whose receive count disagrees with its peer's send count raises
    between posting its buffer and finishing the exchange.  It breaks the
    hub's barrier on the way out, so the peer's exchange ends with an error at
    once instead of waiting for the barrier's timeout.  Host-only: CUDA events
    and streams are replaced by no-op fakes and the buffers are CPU tensors."""
    import contextlib
    import threading
    import time

    import torch
    from hydraphase.partition import ThreadComm
    monkeypatch.setattr(torch.cuda, "Event", _FakeEvent)
    monkeypatch.setattr(torch.cuda, "ExternalStream", _FakeStream)
    monkeypatch.setattr(torch.cuda, "stream", lambda s: contextlib.nullcontext())
    hub = ThreadComm(2, timeout=60.0)
    errors = [None, None]

    def part(rank):
        # part 0 sends 2 cells to part 1; part 1 sends 3 to part 0, which
        # expects 4
        scount = [2] if rank == 0 else [3]
        rcount = [4] if rank == 0 else [2]
        send = torch.zeros(10 * scount[0], dtype=torch.float64)
        recv = torch.zeros(10 * rcount[0], dtype=torch.float64)
        try:
            hub.bind(rank).exchange(send, scount, recv, rcount, [1 - rank], None)
        except Exception as e:      # noqa: BLE001 -- the test inspects it
            errors[rank] = e

    t0 = time.monotonic()
    threads = [threading.Thread(target=part, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=30.0)
    assert not any(t.is_alive() for t in threads)
    assert time.monotonic() - t0 < 10.0
    assert isinstance(errors[0], RuntimeError) and "expects 4 cells" in str(errors[0])
    assert isinstance(errors[1], threading.BrokenBarrierError)


# --- GPU ---------------------------------------------------------------------
def _single(spec, n, prec=PREC_FP64_PARITY):
    with Case(spec.mesh, spec.params(precision=prec)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        d = c.step(n)
        t, cu, gp = c.state()
    return d, cu, gp


def _assert_same(d, cu, gp, ref):
    dr, cur, gpr = ref
    for k in ("time", "dt", "velmag", "diff", "nan_cells"):
        np.testing.assert_array_equal(d[k], dr[k], err_msg=k)
    np.testing.assert_array_equal(cu, cur)
    np.testing.assert_array_equal(gp, gpr)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("nparts", [2, 5, 37])
def test_partitioned_batch_bit_exact(name, nparts):
    from hydraphase.partition import PartitionedCase
    spec = SPECS[name]()
    n = 4
    ref = _single(spec, n)
    P = partition_case(spec, nparts)
    with PartitionedCase(P, spec.params(precision=PREC_FP64_PARITY)) as pc:
        pc.set_state(0.0, spec.cu, spec.ghost_prims)
        d = pc.step(n)
        _, cu, gp = pc.state()
    _assert_same(d, cu, gp, ref)


@pytest.mark.gpu
def test_partitioned_batch_mixed_within_tolerance():
    """The mixed variant evaluates each face once, from the side its face
    list picks; a part may pick the other side, which is the same value up
    to FP32 rounding."""
    from hydraphase.partition import PartitionedCase
    spec = SPECS["cylinder"]()
    _, cu_r, _ = _single(spec, 5, PREC_MIXED)
    P = partition_case(spec, 3)
    with PartitionedCase(P, spec.params(precision=PREC_MIXED)) as pc:
        pc.set_state(0.0, spec.cu, spec.ghost_prims)
        pc.step(5, diagnostics=False)
        _, cu, _ = pc.state()
    rho_r, rho = cu_r[0] + cu_r[5], cu[0] + cu[5]
    assert np.linalg.norm(rho - rho_r) / np.linalg.norm(rho_r) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nparts", [1, 3])
def test_rank_parts_with_thread_exchange_bit_exact(nparts):
    """One handle per part, each stepped by its own host thread; the dt
    minimum and the halo exchange run through hp_set_exchange with
    ThreadComm (stream-ordered copies between the parts' buffers)."""
    import threading

    import torch
    from hydraphase.partition import RankPart, ThreadComm
    spec = SPECS["cylinder"]()
    n = 4
    ref = _single(spec, n)
    torch.cuda.init()
    P = partition_case(spec, nparts)
    hub = ThreadComm(nparts, timeout=60.0)
    parts = [RankPart(P, r, spec.params(precision=PREC_FP64_PARITY), hub.bind(r)) for r in range(nparts)]
    for r, (cp, gp) in enumerate(P.scatter_state(spec.cu, spec.ghost_prims)):
        parts[r].set_state(0.0, cp, gp)
    out, errs = [None] * nparts, []

    def run(r):
        try:
            torch.cuda.set_device(0)
            out[r] = parts[r].step(n)
        except Exception as e:       # reported below
            errs.append(e)
    th = [threading.Thread(target=run, args=(r,)) for r in range(nparts)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    states = [parts[r].state() for r in range(nparts)]
    for p in parts:
        p.close()
    cu, gp = P.gather_state([(s[1], s[2]) for s in states])
    p1 = int(P.owner[0])
    d = {"time": out[0]["time"], "dt": out[0]["dt"], "velmag": out[p1]["velmag"],
         "diff": np.max(np.stack([o["diff"] for o in out]), axis=0),
         "nan_cells": np.sum(np.stack([o["nan_cells"] for o in out]), axis=0)}
    _assert_same(d, cu, gp, ref)


def _nccl_rank(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    from hydraphase.partition import DistComm, RankPart
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    spec = SPECS["cylinder"]()
    ref = _single(spec, 3)
    P = partition_case(spec, 1)
    rp = RankPart(P, 0, spec.params(precision=PREC_FP64_PARITY), DistComm())
    cp, gp = P.scatter_state(spec.cu, spec.ghost_prims)[0]
    rp.set_state(0.0, cp, gp)
    d = rp.step(3)
    _, cu, gpo = rp.state()
    rp.close()
    dist.destroy_process_group()
    same = all(np.array_equal(d[k], ref[0][k]) for k in ("time", "dt", "velmag", "diff")) and \
        np.array_equal(cu, ref[1]) and np.array_equal(gpo, ref[2])
    np.save(os.path.join(out_dir, "nccl.npy"), np.array([same]))


@pytest.mark.gpu
def test_rank_part_dt_allreduce_over_nccl_single_rank(tmp_path):
    """DistComm over NCCL with one rank (one GPU in this run): the library
    calls back at every exchange point and the dt word is allreduced in
    place on the library's stream; the run equals the plain single-mesh
    run bit for bit."""
    mp.spawn(_nccl_rank, args=(1, _free_port(), str(tmp_path)), nprocs=1, join=True)
    assert bool(np.load(tmp_path / "nccl.npy")[0])


@pytest.mark.gpu
def test_halo_and_exchange_argument_errors():
    """hp_set_halo rejects ids out of range, a repeated destination and a
    destination that is also a source, and a table set after the first step;
    hp_set_exchange and hp_set_halo_lists take single-case handles only."""
    import ctypes

    from hydraphase import HP_E_ARG, HP_E_STATE, HP_E_UNSUPPORTED, Batch
    from hydraphase._lib import HP_EXCHANGE_FN, lib
    spec = SPECS["shock_bubble"]()
    P = partition_case(spec, 2)
    L = lib()
    ip = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int32))  # noqa: E731
    with Batch([p.spec.mesh for p in P.parts], spec.params(precision=PREC_FP64_PARITY)) as b:
        dc, de, sc, se = (np.ascontiguousarray(a, np.int32) for a in P.halo_table())
        bad = de.copy()
        bad[0] = 10 ** 7
        assert L.hp_set_halo(b.h, dc.size, ip(dc), ip(bad), ip(sc), ip(se)) == HP_E_ARG
        rep = de.copy()
        rep[1] = rep[0]
        rep_c = dc.copy()
        rep_c[1] = rep_c[0]
        assert L.hp_set_halo(b.h, dc.size, ip(rep_c), ip(rep), ip(sc), ip(se)) == HP_E_ARG
        # a destination that is another entry's source
        d1 = np.array([dc[0], sc[0]], np.int32)
        e1 = np.array([de[0], se[0]], np.int32)
        s1 = np.array([sc[0], dc[0]], np.int32)
        f1 = np.array([se[0], de[0]], np.int32)
        assert L.hp_set_halo(b.h, 2, ip(d1), ip(e1), ip(s1), ip(f1)) == HP_E_ARG
        assert L.hp_set_exchange(b.h, HP_EXCHANGE_FN(lambda u, p, s: None), None) == HP_E_UNSUPPORTED
        assert L.hp_set_halo_lists(b.h, 0, None, 0, None) == HP_E_UNSUPPORTED
        assert L.hp_set_halo(b.h, dc.size, ip(dc), ip(de), ip(sc), ip(se)) == 0
        for c, (cp, gp) in enumerate(P.scatter_state(spec.cu, spec.ghost_prims)):
            b.set_state(c, 0.0, cp, gp)
        b.step(1, diagnostics=False)
        assert L.hp_set_halo(b.h, dc.size, ip(dc), ip(de), ip(sc), ip(se)) == HP_E_STATE
