"""Precision stress: the same case run with FP64 everywhere, with the mixed
variant (FP32 gradients, limiter, reconstruction and fluxes; FP64 state, EOS
and reductions) and with everything in FP32. Each result is compared with
the FP64 one.

The FP64 run uses the parity variant, which is bit-identical to the CPU
oracle (tests/test_gpu_parity.py), so it stands in for the oracle at sizes
and step counts the oracle cannot reach in reasonable time. Reported per
variant:

* relative L2 and max errors of mixture density, pressure and air volume
  fraction, recovered from the conserved state with the reference's
  pressure-equilibrium quadratic (src/sr_primitive.F90:53-91);
* positivity violations: cells with a NaN, a non-positive phase density or
  pressure, or a volume fraction outside [0, 1];
* device time per step.

Two more runs measure the rounding floor, the distance to the FP64 parity
result of a variant that differs from it only by rounding. The FP64 FMA
variant ("fma") is that yardstick: it computes in FP64 throughout and differs
from parity only where the compiler contracts a multiply and an add. Each run
reports the errors of "fma", "mixed" and "fp32" against parity at several step
counts:

* `--stream`: cases of the serving stream (shock-bubble, CFL 0.05), run as one
  batch per variant;
* `--smooth`: the viscous cylinder (O-grid 80x128x16, 983,040 cells, CFL 0.5).

Run as `python -m hydraphase.stress [--steps N] [--size nx,ny,nz] [--stream]
[--smooth]`; prints one JSON object.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from ._lib import PREC_FP32, PREC_FP64, PREC_FP64_PARITY, PREC_MIXED
from .engine import Batch, Case

VARIANTS = (("fp64", PREC_FP64_PARITY), ("mixed", PREC_MIXED), ("fp32", PREC_FP32))


def recover(cu: np.ndarray, flow: dict):
    """Pressure and air volume fraction of a conserved state (10, n)."""
    gg, gp, pinf = flow["gamag"], flow["gamap"], flow["pinf"]
    with np.errstate(all="ignore"):
        eg = cu[4] / cu[0] - 0.5 * (cu[1] ** 2 + cu[2] ** 2 + cu[3] ** 2) / cu[0] ** 2
        ep = cu[9] / cu[5] - 0.5 * (cu[6] ** 2 + cu[7] ** 2 + cu[8] ** 2) / cu[5] ** 2
        bbb = pinf * gp - cu[0] * (gg - 1) * eg - cu[5] * (gp - 1) * ep
        ccc = cu[0] * (gg - 1) * eg * pinf * gp
        pg = (-bbb + np.sqrt(bbb * bbb + 4 * ccc)) * 0.5
        return pg, cu[0] * (gg - 1) * eg / pg


def positivity(cu: np.ndarray, flow: dict) -> dict:
    pg, ag = recover(cu, flow)
    with np.errstate(invalid="ignore"):
        return {"nan_cells": int(np.isnan(cu).any(axis=0).sum()),
                "nonpositive_density": int(((cu[0] <= 0) | (cu[5] <= 0)).sum()),
                "nonpositive_pressure": int((pg <= 0).sum()),
                "alpha_out_of_range": int(((ag < 0) | (ag > 1)).sum())}


def errors(cu: np.ndarray, ref: np.ndarray, flow: dict) -> dict:
    p, a = recover(cu, flow)
    p0, a0 = recover(ref, flow)
    out = {}
    for name, x, y in (("density", cu[0] + cu[5], ref[0] + ref[5]), ("pressure", p, p0), ("alpha_g", a, a0)):
        d = x - y
        with np.errstate(invalid="ignore"):
            out[name] = {"rel_l2": float(np.linalg.norm(d) / max(np.linalg.norm(y), 1e-300)),
                         "max_rel": float(np.nanmax(np.abs(d) / np.maximum(np.abs(y), 1e-300)))
                         if np.isfinite(d).any() else float("nan")}
    return out


def run(spec, steps: int, chunk: int = 100, variants=VARIANTS) -> dict:
    states, out = {}, {}
    for name, prec in variants:
        with Case(spec.mesh, spec.params(precision=prec)) as c:
            c.set_state(0.0, spec.cu, spec.ghost_prims)
            ms, done, first_nan = 0.0, 0, None
            while done < steps:
                n = min(chunk, steps - done)
                ms += c.step_timed(n)
                done += n
                _, cu, _ = c.state()
                if first_nan is None and np.isnan(cu).any():
                    first_nan = done
            states[name] = cu
            out[name] = {"ms_per_step": ms / steps, "first_nan_by_step": first_nan,
                         "positivity": positivity(cu, spec.flow)}
    for name, _ in variants:
        if name != "fp64":
            out[name]["error_vs_fp64"] = errors(states[name], states["fp64"], spec.flow)
    return out


FLOOR_VARIANTS = (("fma", PREC_FP64), ("mixed", PREC_MIXED), ("fp32", PREC_FP32))


def _summarise(errs: list) -> dict:
    """Median and maximum over cases of the density and alpha_g errors."""
    out = {}
    for q in ("density", "alpha_g"):
        v = [e[q]["rel_l2"] for e in errs]
        out[q] = {"median": float(np.median(v)), "max": float(np.max(v))}
    return out


def floor_batch(specs, checkpoints=(10, 100, 500, 1000), variants=FLOOR_VARIANTS) -> dict:
    """Run every case of `specs` as one batch per variant, FP64 parity
    first, and report each variant's errors against parity at every
    checkpoint (median and maximum over the cases)."""
    states = {}
    for name, prec in (("fp64", PREC_FP64_PARITY),) + tuple(variants):
        with Batch([sp.mesh for sp in specs], specs[0].params(precision=prec)) as b:
            for k, sp in enumerate(specs):
                b.set_state(k, 0.0, sp.cu, sp.ghost_prims)
            done, snaps = 0, []
            for c in checkpoints:
                b.step(c - done, diagnostics=False)
                done = c
                snaps.append([b.state(k)[1] for k in range(len(specs))])
            states[name] = snaps
    out = {}
    for name, _ in variants:
        out[name] = {str(c): _summarise([errors(states[name][i][k], states["fp64"][i][k], specs[k].flow)
                                         for k in range(len(specs))])
                     for i, c in enumerate(checkpoints)}
    return out


def main():
    from . import cases
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--size", default="60,60,90", help="hexes nx,ny,nz of the box (6 tets each)")
    ap.add_argument("--stream", action="store_true", help="rounding floor on 16 serving-stream cases")
    ap.add_argument("--smooth", action="store_true", help="rounding floor on the viscous cylinder")
    a = ap.parse_args()
    if a.stream or a.smooth:
        res = {}
        if a.stream:
            reqs = cases.serving_stream(n_cases=16, steps=1000, cells=(6000, 100000), seed=5)
            res["stream"] = {"workload": "16 serving-stream shock-bubble cases, 6k-100k cells, CFL 0.05, "
                                         "SSP-RK3 (seed 5)",
                             **floor_batch([r.spec for r in reqs])}
        if a.smooth:
            sp = cases.cylinder(nr=80, nt=128, nz=16, seed=1, alpha_w_drop=1e-5, alpha_w_bg=1e-6)
            res["smooth"] = {"workload": f"viscous cylinder O-grid 80x128x16, {sp.mesh.neles} cells, CFL 0.5, "
                                         "SSP-RK3", **floor_batch([sp])}
        print(json.dumps(res))
        return
    nx, ny, nz = (int(v) for v in a.size.split(","))
    spec = cases.shock_lattice(nx=nx, ny=ny, nz=nz)
    res = {"workload": f"shock lattice: {spec.mesh.neles} cells, 5e9 Pa water shock on a 5x5 air-bubble "
                       f"lattice, SSP-RK3, CFL {spec.flow['cfl']}, {a.steps} steps",
           "cells": spec.mesh.neles, "steps": a.steps, **run(spec, a.steps)}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
