"""Serving many cases on one GPU: continuous admission against an HBM budget.

The reference runs one case per process. Here a request loop takes cases
(mesh + initial state + step count) as they arrive, keeps each case's mesh
and solution resident on the device, and advances all admitted cases
together:

* **Admission.** It is FIFO. A case is admitted as soon as a slot is free
  (at most `max_active` cases in flight) and its device bytes
  (`hp_estimate_bytes`) fit in what is left of `hbm_budget`.
* **Set-up.** Host-side geometry, layout and upload (`hp_create` +
  `hp_set_state`) run on a pool of worker threads. They overlap with the
  device work of the cases already running.
* **Overlap.** Every case owns a CUDA stream and replays its step as a CUDA
  graph. The loop enqueues `chunk` steps on a case whenever its previous
  chunk is done (`hp_poll`, non-blocking). So the kernels of different cases
  overlap on the device, and a case that arrives later joins at the next
  chunk boundary without waiting for the others.
* **Completion.** When a case has run all its steps, its state is copied back
  to the host, its device memory is released (stream-ordered, with no
  device-wide synchronisation), and its slot and bytes are freed for the
  queue.

Time-to-solution is measured from arrival to the result on the host,
queueing included. A case's result does not depend on what else runs: each
case has its own buffers, stream and reductions, and the kernels are
deterministic. tests/test_serving.py checks this bit for bit.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from ._lib import PREC_MIXED, HydraError
from .engine import Case, estimate_bytes


@dataclass
class CaseResult:
    rid: int
    cells: int
    steps: int
    arrival: float          # s from the stream's start
    admitted: float         # admission decision (set-up starts)
    started: float          # first chunk enqueued
    finished: float         # state back on the host
    device_bytes: int
    time: float = 0.0       # simulation time reached
    cu: np.ndarray | None = None
    ghost_prims: np.ndarray | None = None
    error: str | None = None  # set-up failure (e.g. HP_E_NOMEM), no result

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Active:
    req: object
    case: Case
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

    def summary(self) -> dict:
        ok = [r for r in self.results if r.error is None]
        lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
        upd = sum(r.cells * 3 * r.steps for r in ok)
        return {"cases": len(ok), "failed": len(self.results) - len(ok), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "makespan_s": self.makespan, "updates_per_s": upd / self.makespan if self.makespan else 0.0,
                "peak_device_bytes": self.peak_bytes, "peak_active": self.peak_active}


class Server:
    """Continuous-batching request loop over per-case handles.

    requests: objects with .rid, .arrival (s), .steps, .spec (a CaseSpec)
    precision: HP_PREC_* of every case
    hbm_budget: device bytes the admitted cases may hold together
    max_active: cases in flight (set up or running)
    chunk: steps enqueued per case per turn of the loop
    keep_state: copy each final state back (False keeps only the timing)
    """

    def __init__(self, hbm_budget: int, precision: int = PREC_MIXED, max_active: int = 12, chunk: int = 25,
                 setup_workers: int = 4, keep_state: bool = True, param_overrides: dict | None = None):
        self.budget = int(hbm_budget)
        self.precision = precision
        self.max_active = max_active
        self.chunk = chunk
        self.workers = setup_workers
        self.keep_state = keep_state
        self.over = dict(param_overrides or {})

    def _params(self, spec):
        return spec.params(precision=self.precision, **self.over)

    @staticmethod
    def _setup(spec, params):
        c = Case(spec.mesh, params)
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        return c

    def run(self, requests, realtime: bool = True) -> ServeReport:
        """Serve `requests`; with realtime=False every case arrives at t=0."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list = []
        setting_up: list = []      # (future, req, bytes, t_admit)
        active: list[_Active] = []
        rep = ServeReport()
        used = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        with ThreadPoolExecutor(self.workers) as pool:
            while pending or queue or setting_up or active:
                progressed = False
                t = now()
                while pending and (not realtime or pending[0].arrival <= t):
                    queue.append(pending.pop(0))
                    progressed = True
                # FIFO admission against slots and bytes
                while queue and len(setting_up) + len(active) < self.max_active:
                    req = queue[0]
                    p = self._params(req.spec)
                    b = estimate_bytes(req.spec.mesh, p)
                    if used + b > self.budget and (setting_up or active):
                        break
                    queue.pop(0)
                    used += b
                    rep.peak_bytes = max(rep.peak_bytes, used)
                    setting_up.append((pool.submit(self._setup, req.spec, p), req, b, now()))
                    progressed = True
                # cases whose set-up finished start stepping
                still = []
                for fut, req, b, ta in setting_up:
                    if fut.done():
                        try:
                            case = fut.result()
                        except HydraError as e:
                            used -= b
                            rep.results.append(CaseResult(req.rid, req.spec.mesh.neles, req.steps, req.arrival,
                                                          ta, ta, now(), b, error=str(e)))
                            progressed = True
                            continue
                        n = min(self.chunk, req.steps)
                        case.step(n, diagnostics=False)
                        active.append(_Active(req, case, b, ta, now(), req.steps - n))
                        progressed = True
                    else:
                        still.append((fut, req, b, ta))
                setting_up = still
                rep.peak_active = max(rep.peak_active, len(active) + len(setting_up))
                # next chunk for every case whose previous chunk is done
                keep = []
                for a in active:
                    if a.case.poll():
                        keep.append(a)
                        continue
                    progressed = True
                    if a.remaining > 0:
                        n = min(self.chunk, a.remaining)
                        a.case.step(n, diagnostics=False)
                        a.remaining -= n
                        keep.append(a)
                        continue
                    tm, cu, gp = a.case.state() if self.keep_state else (0.0, None, None)
                    a.case.close()
                    used -= a.bytes
                    rep.results.append(CaseResult(a.req.rid, a.req.spec.mesh.neles, a.req.steps, a.req.arrival,
                                                  a.admitted, a.started, now(), a.bytes, tm, cu, gp))
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
