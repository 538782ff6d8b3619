"""Autotuner: measures, on the GPU in use, the launch and serving settings
for each mesh-size class, and caches the choices.

Two levels are tuned:

* **Kernels** (`tune_block_size`, `tune_face_mode`, `tune_step_mode`). These are the threads
  per block of the one-thread-per-cell kernels (primitive recovery, JST
  smoothing, ghost fill, and the gradients and face gathers of the
  FP32-arithmetic variants) and, for those variants, how the HLLC fluxes
  reach the cells: once per face with the face records gathered per cell in
  face order (mode 0), once from each side with four lanes per cell (mode 1,
  one kernel fewer per stage), once per face added to per-cell sums colour by
  colour so that no two faces of a launch share a cell (mode 2: colouring, no
  atomics, a fixed order) or, when the caller accepts sums whose last bits
  vary between runs, with atomic adds (mode 3). Every candidate runs device-timed steps (CUDA
  events) of a representative case of the class: the best of three runs from
  the initial state, each of at least 20 ms (up to 200 steps).  The fastest
  is kept. The four-lane kernels have their block size fixed by their launch
  bounds, tuned per precision variant at build time. Last, whether a step
  replays its ~20 kernels from a CUDA graph or runs as one fused cooperative
  kernel (grid-wide barriers between the phases), which saves the fixed
  cost of the launches on small meshes.
* **Serving** (`tune_serving`). These are the units in flight, the
  multi-mesh batch size and the steps enqueued per turn. Every candidate
  serves a short sample of the stream with all cases arriving at once, and
  the one with the highest throughput is kept.

Results are stored in a JSON file keyed by GPU name, precision and size
class. By default it is ~/.cache/hydraphase/tune.json; the
HYDRAPHASE_TUNE_CACHE environment variable overrides the path. Later runs
read the cache instead of measuring again.
"""
from __future__ import annotations

import json
import math
import os
import time

from ._lib import PREC_FP32, PREC_FP64_PARITY, PREC_MIXED
from .engine import Case

SIZE_CLASSES = ((0, 20000, "xs"), (20000, 100000, "s"), (100000, 400000, "m"), (400000, 1 << 62, "l"))
BLOCK_CANDIDATES = (64, 128, 256, 512)


def size_class(cells: int) -> str:
    for lo, hi, name in SIZE_CLASSES:
        if lo <= cells < hi:
            return name
    return SIZE_CLASSES[-1][2]


def cache_path() -> str:
    return os.environ.get("HYDRAPHASE_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "hydraphase", "tune.json"))


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(data: dict) -> None:
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _key(precision: int, cls: str, what: str) -> str:
    return f"{_gpu_name()}|prec{precision}|{cls}|{what}"


def _ms_per_step(c, spec, steps: int, min_ms: float = 20.0, max_steps: int = 200, repeats: int = 3) -> float:
    """Device ms per step of an open Case: the best of `repeats` timed runs
    from the initial state, each of at least `steps` steps and, up to
    max_steps, of at least min_ms in all.  Small meshes step in a fraction of
    a millisecond, where a few steps time mostly launch noise and the choice
    between candidates would be a coin toss."""
    c.set_state(0.0, spec.cu, spec.ghost_prims)
    c.step(2, diagnostics=False)
    probe = c.step_timed(steps) / steps
    n = min(max_steps, max(steps, int(math.ceil(min_ms / max(probe, 1e-3)))))
    best = float("inf")
    for _ in range(repeats):
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.step(1, diagnostics=False)
        best = min(best, c.step_timed(n) / n)
    return best


def tune_block_size(spec, precision: int = PREC_MIXED, candidates=BLOCK_CANDIDATES, steps: int = 6,
                    use_cache: bool = True) -> tuple[int, dict]:
    """Threads per block of the per-cell kernels for the size class of
    `spec`; returns (best, {candidate: ms per step})."""
    key = _key(precision, size_class(spec.mesh.neles), "block_size")
    if use_cache:
        hit = _load().get(key)
        if hit:
            return int(hit["best"]), {int(k): v for k, v in hit["ms"].items()}
    ms = {}
    for b in candidates:
        with Case(spec.mesh, spec.params(precision=precision, block_size=int(b))) as c:
            ms[int(b)] = _ms_per_step(c, spec, steps)
    best = min(ms, key=ms.get)
    data = _load()
    data[key] = {"best": best, "ms": {str(k): v for k, v in ms.items()}, "cells": spec.mesh.neles,
                 "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(data)
    return best, ms


def tune_face_mode(spec, precision: int = PREC_MIXED, block_size: int = 0, steps: int = 6,
                   use_cache: bool = True, deterministic: bool = True) -> tuple[int, dict]:
    """hp_params.face_mode for the size class of `spec` in the
    FP32-arithmetic variants: 0 (once per face, records gathered per cell),
    1 (once from each side), 2 (once per face, per-cell sums colour by
    colour) and, unless `deterministic`, 3 (once per face, atomic sums, whose
    last bits vary between runs); returns (best, {mode: ms per step}).  The
    FP64 variants have one mode."""
    if precision not in (PREC_MIXED, PREC_FP32):
        return 0, {}
    modes = (0, 1, 2) if deterministic else (0, 1, 2, 3)
    key = _key(precision, size_class(spec.mesh.neles), f"face_mode_b{block_size}" + ("" if deterministic else "_a"))
    if use_cache:
        hit = _load().get(key)
        if hit:
            return int(hit["best"]), {int(k): v for k, v in hit["ms"].items()}
    ms = {}
    for mode in modes:
        with Case(spec.mesh, spec.params(precision=precision, block_size=int(block_size), face_mode=mode)) as c:
            ms[mode] = _ms_per_step(c, spec, steps)
    best = min(ms, key=ms.get)
    data = _load()
    data[key] = {"best": best, "ms": {str(k): v for k, v in ms.items()}, "cells": spec.mesh.neles,
                 "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(data)
    return best, ms


def tune_step_mode(spec, precision: int = PREC_MIXED, block_size: int = 0, face_mode: int = 0, steps: int = 6,
                   use_cache: bool = True) -> tuple[int, dict]:
    """hp_params.use_graph for the size class of `spec`: 1 (the step's
    kernels replayed from a CUDA graph) or 2 (the fused step, one
    cooperative kernel per step); returns (best, {mode: ms per step}).
    Only the FP64 parity variant has the fused step (the variants built with
    FMA contraction keep the graph), so the others return (1, {})."""
    if precision != PREC_FP64_PARITY:
        return 1, {}
    key = _key(precision, size_class(spec.mesh.neles), f"step_mode_b{block_size}_f{face_mode}")
    if use_cache:
        hit = _load().get(key)
        if hit:
            return int(hit["best"]), {int(k): v for k, v in hit["ms"].items()}
    ms = {}
    for mode in (1, 2):
        with Case(spec.mesh, spec.params(precision=precision, block_size=int(block_size), face_mode=int(face_mode),
                                         use_graph=mode)) as c:
            ms[mode] = _ms_per_step(c, spec, steps)
    best = min(ms, key=ms.get)
    data = _load()
    data[key] = {"best": best, "ms": {str(k): v for k, v in ms.items()}, "cells": spec.mesh.neles,
                 "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(data)
    return best, ms


def tune_serving(sample, precision: int = PREC_MIXED, hbm_budget: int = 150 << 30, grid=None, steps: int = 20,
                 use_cache: bool = True) -> tuple[dict, list]:
    """Serving settings (max_active, batch_cells, chunk) for a sample of the
    stream (a list of requests), each case run for `steps` steps with every
    case arriving at once; returns (best, [(settings, updates/s), ...])."""
    from .serve import Server
    mean_cells = int(sum(r.spec.mesh.neles for r in sample) / max(len(sample), 1))
    key = _key(precision, size_class(mean_cells), "serving")
    if use_cache:
        hit = _load().get(key)
        if hit:
            return hit["best"], hit["trials"]
    grid = grid or [dict(max_active=m, batch_cells=b, chunk=c)
                    for m in (8, 16, 32) for b in (0, 200000) for c in (10, 25)]
    trials = []
    short = [type(r)(r.rid, 0.0, steps, r.spec) for r in sample]
    for g in grid:
        rep = Server(hbm_budget, precision=precision, keep_state=False, **g).run(short, realtime=False)
        trials.append((g, rep.summary()["updates_per_s"]))
    best = max(trials, key=lambda t: t[1])[0]
    data = _load()
    data[key] = {"best": best, "trials": trials, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(data)
    return best, trials
