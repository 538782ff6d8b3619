"""Serving many cases on one GPU: continuous admission against an HBM budget.

The reference runs one case per process. Here a request loop takes cases
(mesh + initial state + step count) as they arrive, keeps each case's mesh
and solution resident on the device, and advances all admitted cases
together:

* **Admission.** It is FIFO. A unit (one case or a batch of them) is
  admitted as soon as a slot is free (at most `max_active` units in flight)
  and its device bytes (`hp_estimate_bytes` / `hp_estimate_batch_bytes`) fit
  in what is left of `hbm_budget`.
* **Batching.** With `batch_cells` set, consecutive queued cases smaller than
  that, with equal parameters and step counts, are set up together as one
  multi-mesh batch (`hp_create_batch`) of at most `batch_cells` cells. Each
  kernel launch of a step then sweeps all of them.
* **Set-up.** Host-side geometry, layout and upload (`hp_create` +
  `hp_set_state`) run on a pool of worker threads. They overlap with the
  device work of the units already running.
* **Overlap.** Every unit owns a CUDA stream and replays its step as a CUDA
  graph. The loop enqueues `chunk` steps on a unit whenever its previous
  chunk is done (`hp_poll`, non-blocking). So the kernels of different units
  overlap on the device, and a case that arrives later joins at the next
  chunk boundary without waiting for the others.
* **Completion.** When a unit has run all its steps, its states are copied
  back to the host, its device memory is released (stream-ordered, with no
  device-wide synchronisation), and its slot and bytes are freed for the
  queue.

Time-to-solution is measured from arrival to the result on the host,
queueing included. A case's result does not depend on what else runs: each
unit has its own buffers, stream and reductions, the members of a batch keep
their own scalars, and the kernels are deterministic. tests/test_serving.py
checks this bit for bit.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from ._lib import PREC_MIXED, HydraError
from .engine import Batch, Case, estimate_batch_bytes, estimate_bytes


@dataclass
class CaseResult:
    rid: int
    cells: int
    steps: int
    arrival: float          # s from the stream's start
    admitted: float         # admission decision (set-up starts)
    started: float          # first chunk enqueued
    finished: float         # state back on the host
    device_bytes: int       # of its unit, shared evenly by a batch's members
    time: float = 0.0       # simulation time reached
    cu: np.ndarray | None = None
    ghost_prims: np.ndarray | None = None
    error: str | None = None  # set-up failure (e.g. HP_E_NOMEM), no result

    @property
    def nan_cells(self) -> int:
        """Cells whose final state holds a NaN (-1 without a kept state)."""
        return -1 if self.cu is None else int(np.isnan(self.cu).any(axis=0).sum())

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Active:
    reqs: list             # the requests of this unit (one case or a batch)
    handle: object         # Case or Batch
    bytes: int
    admitted: float
    started: float
    remaining: int


@dataclass
class ServeReport:
    results: list = field(default_factory=list)
    makespan: float = 0.0
    peak_bytes: int = 0
    peak_active: int = 0
    units: int = 0

    def summary(self) -> dict:
        ok = [r for r in self.results if r.error is None]
        lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
        upd = sum(r.cells * 3 * r.steps for r in ok)
        return {"cases": len(ok), "failed": len(self.results) - len(ok), "units": self.units,
                "cases_with_nan": sum(1 for r in ok if r.nan_cells > 0),
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean()), "makespan_s": self.makespan,
                "updates_per_s": upd / self.makespan if self.makespan else 0.0,
                "peak_device_bytes": self.peak_bytes, "peak_active": self.peak_active}


def _same_setup(a, b) -> bool:
    return a.steps == b.steps and a.spec.flow == b.spec.flow and a.spec.extra == b.spec.extra


class Server:
    """Continuous-batching request loop over per-unit handles.

    requests: objects with .rid, .arrival (s), .steps, .spec (a CaseSpec)
    precision: HP_PREC_* of every case
    hbm_budget: device bytes the admitted units may hold together
    max_active: units in flight (set up or running)
    chunk: steps enqueued per unit per turn of the loop
    chunk_cell_steps: if set, a unit of c cells gets max(chunk,
        chunk_cell_steps // c) steps per turn, so small units go back to the
        host loop no more often than large ones
    setup_workers: host threads running hp_create + hp_set_state; with 4,
        the 48-case stream of the benchmark queued for set-up (median wait
        1.8 s), with 8 it did not (0.1 s)
    keep_state: copy each final state back (False keeps only the timing)
    batch_cells: cases below this size are grouped into multi-mesh batches of
        at most this many cells (0: every case on its own handle)
    max_batch: cases per batch at most
    block_size: threads per block of the per-cell kernels: an int, a dict
        from hydraphase.tune.size_class() to an int, or None (256)
    face_mode: hp_params.face_mode, an int or a dict by size class (None: 0)
    step_mode: hp_params.use_graph (1: graph, 2: fused step), an int or a
        dict by size class (None: 1)
    host_threads: OpenMP threads of each set-up worker's hp_create (None: the
        cores divided among the workers, so that concurrent set-ups do not
        oversubscribe the host and delay the loop that feeds the GPU)
    """

    def __init__(self, hbm_budget: int, precision: int = PREC_MIXED, max_active: int = 12, chunk: int = 25,
                 setup_workers: int = 8, keep_state: bool = True, param_overrides: dict | None = None,
                 batch_cells: int = 0, max_batch: int = 64, block_size=None, face_mode=None,
                 chunk_cell_steps: int | None = None, host_threads: int | None = None, step_mode=None):
        self.budget = int(hbm_budget)
        self.precision = precision
        self.max_active = max_active
        self.chunk = chunk
        self.workers = setup_workers
        self.keep_state = keep_state
        self.over = dict(param_overrides or {})
        self.batch_cells = int(batch_cells)
        self.max_batch = int(max_batch)
        self.block_size = block_size
        self.face_mode = face_mode
        self.step_mode = step_mode
        self.chunk_cell_steps = chunk_cell_steps
        self.host_threads = host_threads

    def _params(self, spec, cells: int):
        from .tune import size_class
        over = dict(self.over)
        b, fm = self.block_size, self.face_mode
        if isinstance(b, dict):
            b = b.get(size_class(cells))
        if isinstance(fm, dict):
            fm = fm.get(size_class(cells))
        if b and "block_size" not in over:
            over["block_size"] = int(b)
        if fm and "face_mode" not in over:
            over["face_mode"] = int(fm)
        sm = self.step_mode
        if isinstance(sm, dict):
            sm = sm.get(size_class(cells))
        if sm and "use_graph" not in over:
            over["use_graph"] = int(sm)
        return spec.params(precision=self.precision, **over)

    @staticmethod
    def _setup(unit, params):
        if len(unit) == 1:
            spec = unit[0].spec
            c = Case(spec.mesh, params)
            c.set_state(0.0, spec.cu, spec.ghost_prims)
            return c
        b = Batch([r.spec.mesh for r in unit], params)
        for k, r in enumerate(unit):
            b.set_state(k, 0.0, r.spec.cu, r.spec.ghost_prims)
        return b

    def _chunk_for(self, unit) -> int:
        """Steps per turn for a unit (its cases' total cells)."""
        if not self.chunk_cell_steps:
            return self.chunk
        cells = sum(r.spec.mesh.neles for r in unit)
        return max(self.chunk, int(self.chunk_cell_steps) // max(cells, 1))

    def _take_unit(self, queue):
        """The next unit from the head of the queue: one case, or the longest
        run of small compatible cases that fits in batch_cells."""
        head = queue[0]
        cells = head.spec.mesh.neles
        if not self.batch_cells or cells >= self.batch_cells:
            return [head]
        unit = [head]
        for r in queue[1:]:
            n = r.spec.mesh.neles
            if len(unit) >= self.max_batch or cells + n > self.batch_cells or not _same_setup(head, r):
                break
            unit.append(r)
            cells += n
        return unit

    def run(self, requests, realtime: bool = True) -> ServeReport:
        """Serve `requests`; with realtime=False every case arrives at t=0."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list = []
        setting_up: list = []      # (future, unit, bytes, t_admit)
        active: list[_Active] = []
        rep = ServeReport()
        used = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        import os
        from ._lib import lib
        nthr = self.host_threads if self.host_threads is not None else max(1, (os.cpu_count() or 1) // self.workers)
        with ThreadPoolExecutor(self.workers, initializer=lambda: lib().hp_set_host_threads(int(nthr))) as pool:
            while pending or queue or setting_up or active:
                progressed = False
                t = now()
                while pending and (not realtime or pending[0].arrival <= t):
                    queue.append(pending.pop(0))
                    progressed = True
                # FIFO admission against slots and bytes
                while queue and len(setting_up) + len(active) < self.max_active:
                    unit = self._take_unit(queue)
                    cells = sum(r.spec.mesh.neles for r in unit)
                    p = self._params(unit[0].spec, cells)
                    b = estimate_bytes(unit[0].spec.mesh, p) if len(unit) == 1 else \
                        estimate_batch_bytes([r.spec.mesh for r in unit], p)
                    if used + b > self.budget and (setting_up or active):
                        break
                    del queue[:len(unit)]
                    used += b
                    rep.peak_bytes = max(rep.peak_bytes, used)
                    rep.units += 1
                    setting_up.append((pool.submit(self._setup, unit, p), unit, b, now()))
                    progressed = True
                # units whose set-up finished start stepping
                still = []
                for fut, unit, b, ta in setting_up:
                    if not fut.done():
                        still.append((fut, unit, b, ta))
                        continue
                    progressed = True
                    try:
                        handle = fut.result()
                    except HydraError as e:
                        used -= b
                        for r in unit:
                            rep.results.append(CaseResult(r.rid, r.spec.mesh.neles, r.steps, r.arrival, ta, ta,
                                                          now(), b // len(unit), error=str(e)))
                        continue
                    n = min(self._chunk_for(unit), unit[0].steps)
                    handle.step(n, diagnostics=False)
                    active.append(_Active(unit, handle, b, ta, now(), unit[0].steps - n))
                setting_up = still
                rep.peak_active = max(rep.peak_active, len(active) + len(setting_up))
                # next chunk for every unit whose previous chunk is done
                keep = []
                for a in active:
                    if a.handle.poll():
                        keep.append(a)
                        continue
                    progressed = True
                    if a.remaining > 0:
                        n = min(self._chunk_for(a.reqs), a.remaining)
                        a.handle.step(n, diagnostics=False)
                        a.remaining -= n
                        keep.append(a)
                        continue
                    batch = isinstance(a.handle, Batch)
                    for k, r in enumerate(a.reqs):
                        if self.keep_state:
                            tm, cu, gp = a.handle.state(k) if batch else a.handle.state()
                        else:
                            tm, cu, gp = 0.0, None, None
                        rep.results.append(CaseResult(r.rid, r.spec.mesh.neles, r.steps, r.arrival, a.admitted,
                                                      a.started, now(), a.bytes // len(a.reqs), tm, cu, gp))
                    a.handle.close()
                    used -= a.bytes
                active = keep
                if not progressed:
                    time.sleep(0.0002)
        rep.makespan = now()
        rep.results.sort(key=lambda r: r.rid)
        return rep


def run_alone(spec, steps: int, precision: int = PREC_MIXED, param_overrides: dict | None = None):
    """The same case on its own (reference result for the mixed-stream test)."""
    with Case(spec.mesh, spec.params(precision=precision, **(param_overrides or {}))) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.step(steps, diagnostics=False)
        return c.state()
