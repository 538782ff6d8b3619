"""Host logic of the serving loop (hydraphase.serve.Server) on the CPU.

The engine's handles are replaced by fakes that record what the loop asks of
them, so admission, batching, chunking and failure handling are checked
without a GPU:

* FIFO admission never holds more units than `max_active` nor more
  estimated bytes than the HBM budget (one unit may exceed an empty budget);
* small compatible cases are grouped into batches of at most `batch_cells`;
* every case runs exactly its step count, in chunks of `chunk` steps, or of
  `chunk_cell_steps / cells` steps for small units;
* a unit whose set-up fails reports the error for each of its cases, gives
  its bytes back, and the others still finish.
"""
import threading

import numpy as np
import pytest

import hydraphase.serve as serve
from hydraphase import HP_E_NOMEM, HydraError, cases
from hydraphase.cases import StreamCase

BYTES_PER_CELL = 1000


class FakeHandle:
    """Stands in for Case/Batch: steps finish after two polls."""
    lock = threading.Lock()
    live = 0
    peak_live = 0
    fail_cells = set()

    def __init__(self, meshes, params):
        self.cells = [m.neles for m in meshes]
        if sum(self.cells) in FakeHandle.fail_cells:
            raise HydraError(HP_E_NOMEM, "fake out of memory")
        self.steps = 0
        self.chunks = []
        self.busy = 0
        with FakeHandle.lock:
            FakeHandle.live += 1
            FakeHandle.peak_live = max(FakeHandle.peak_live, FakeHandle.live)

    def set_state(self, *a):
        pass

    def step(self, n, diagnostics=False):
        self.steps += n
        self.chunks.append(n)
        self.busy = 2

    def poll(self):
        self.busy -= 1
        return self.busy > 0

    def state(self, k=0):
        return float(self.steps), np.zeros((10, self.cells[k])), np.zeros((6, 0))

    def close(self):
        with FakeHandle.lock:
            FakeHandle.live -= 1
        RECORD.append(self)


class FakeCase(FakeHandle):
    def __init__(self, mesh, params):
        super().__init__([mesh], params)


class FakeBatch(FakeHandle):
    def set_state(self, c, *a):
        pass


RECORD: list = []


@pytest.fixture
def fake_engine(monkeypatch):
    RECORD.clear()
    FakeHandle.live = FakeHandle.peak_live = 0
    FakeHandle.fail_cells = set()
    monkeypatch.setattr(serve, "Case", FakeCase)
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    monkeypatch.setattr(serve, "estimate_bytes", lambda mesh, p: mesh.neles * BYTES_PER_CELL)
    monkeypatch.setattr(serve, "estimate_batch_bytes",
                        lambda meshes, p: sum(m.neles for m in meshes) * BYTES_PER_CELL)
    return RECORD


def _stream(sizes, steps=60):
    meshes = {}
    out = []
    for k, n in enumerate(sizes):
        if n not in meshes:
            meshes[n] = cases.shock_bubble(n=n, alpha_min=0.1)
        out.append(StreamCase(k, 0.0, steps, meshes[n]))
    return out


def test_all_cases_finish_in_order(fake_engine):
    reqs = _stream([2, 3, 2, 4, 3])
    rep = serve.Server(1 << 40, max_active=3, chunk=25, keep_state=True).run(reqs, realtime=False)
    assert [r.rid for r in rep.results] == list(range(5))
    assert all(r.error is None and r.steps == 60 for r in rep.results)
    assert all(r.cu.shape == (10, req.spec.mesh.neles) for r, req in zip(rep.results, reqs))
    assert all(h.steps == 60 and h.chunks == [25, 25, 10] for h in fake_engine)
    assert rep.peak_active <= 3 and FakeHandle.live == 0


def test_budget_and_slots_bound_admission(fake_engine):
    reqs = _stream([3, 3, 3, 3])
    cell_bytes = reqs[0].spec.mesh.neles * BYTES_PER_CELL
    rep = serve.Server(int(1.5 * cell_bytes), max_active=4, keep_state=False).run(reqs, realtime=False)
    assert rep.peak_bytes <= 1.5 * cell_bytes and FakeHandle.peak_live == 1
    assert len(rep.results) == 4 and all(r.error is None for r in rep.results)
    rep = serve.Server(1 << 40, max_active=2, keep_state=False).run(reqs, realtime=False)
    assert rep.peak_active <= 2


def test_small_cases_are_batched(fake_engine):
    reqs = _stream([2, 2, 2, 2, 4])           # 48-cell cases, then a 384-cell case
    small = reqs[0].spec.mesh.neles
    rep = serve.Server(1 << 40, max_active=8, batch_cells=3 * small, keep_state=True).run(reqs, realtime=False)
    units = sorted(tuple(h.cells) for h in fake_engine)
    assert units == sorted([(small,) * 3, (small,), (reqs[4].spec.mesh.neles,)])
    assert rep.units == 3 and all(r.error is None for r in rep.results)


def test_chunks_scale_with_unit_size(fake_engine):
    reqs = _stream([2, 4], steps=100)
    srv = serve.Server(1 << 40, max_active=4, chunk=10, chunk_cell_steps=2000, keep_state=False)
    assert srv._chunk_for([reqs[0]]) == max(10, 2000 // reqs[0].spec.mesh.neles)
    assert srv._chunk_for([reqs[1]]) == 10
    srv.run(reqs, realtime=False)
    by_cells = {h.cells[0]: h.chunks for h in fake_engine}
    assert by_cells[reqs[0].spec.mesh.neles][0] == 2000 // reqs[0].spec.mesh.neles
    assert by_cells[reqs[1].spec.mesh.neles] == [10] * 10


def test_setup_failure_reported_and_bytes_released(fake_engine):
    reqs = _stream([2, 3, 2])
    FakeHandle.fail_cells = {reqs[1].spec.mesh.neles}
    rep = serve.Server(1 << 40, max_active=1, keep_state=False).run(reqs, realtime=False)
    errs = {r.rid: r.error for r in rep.results}
    assert errs[0] is None and errs[2] is None and "fake out of memory" in errs[1]
    assert rep.summary()["failed"] == 1 and rep.summary()["cases"] == 2
