#!/usr/bin/env python
"""Throughput benchmark of the residual-and-update step (one JSON line).

Metric: cell-RK-stage updates/s = active cells x RK stages x steps / device
time of the step loop, the reference solver's throughput measure.

Workload (N=1): viscous air flow past a cylinder, O-grid 160 x 256 x 20 hexes
split into 6 tets (4,915,200 cells), Mach 0.3, Re_D 150, SSP-RK3, CFL 0.25,
32 water-rich droplets; synthetic, generated in the reference's formats.
Every rank runs its own replica (the path does not shard across GPUs here):
value = cells x stages x steps summed over ranks / max-over-ranks time.

Arms:
  default          the CUDA engine through its C ABI (libhydraphase.so)
  --impl reference the reference algorithm on the host cores (the FP64 CPU
                   restatement in oracle/, since the Fortran reference cannot
                   be built here), on the same workload and step counts.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "multiphase-code_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "cell-RK-stage updates/s, mixed vs FP64 CUDA at stated L2 err; p50/p99 case latency"
UNIT = "cell-stage/s"

# Compulsory bytes per cell and RK stage (each array crossing HBM once):
# the whole step in FP64 and in the mixed variant.
STEP_BYTES_FP64 = 772
STEP_BYTES_MIXED = 566


def flux_kernel_bytes(grad_bytes: int, rk_scheme: int) -> float:
    """Bytes the fused flux + source + RK-update kernel must move per cell:
    14 primitives, 33 gradient components, phi, centroid, vol, dl, 12 face
    vectors, 12 face centroids, 4 neighbour ids, face kinds, iblank, d24 (10),
    vis (8), cu (10) read; cn (10) written; cn read on stages 2.. and cn1
    traffic of the reference scheme, averaged over the stages."""
    reads = 14 * 8 + 33 * grad_bytes + 8 + 24 + 16 + 96 + 96 + 16 + 4 + 4 + 80 + 64 + 80
    if rk_scheme == 1:
        reads += 80 * 2 / 3
        writes = 80
    else:
        reads += 80 * 3 / 4 + 80 / 4
        writes = 80 + 80 / 4
    return reads + writes


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open(self.out.name).read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CFL of the cylinder workloads. The reference's time step is convective
# only (src/main.F90:541-555), and with it the near-wall cells of this O-grid
# (0.005D spacing, Re_D 150) go unstable at CFL 0.5 after 150-200 steps (NaN
# from the wall outwards), while CFL 0.25 runs 1000 steps. The cost of a step
# does not depend on the CFL.
CYL_CFL = 0.25
# FP64 wall layers of the second mixed measurement (hp_params.wall_fp64_layers):
# breadth-first tet layers from the cylinder wall.  On this mesh 80 layers is
# the smallest count whose density error after 1000 steps equals that of the
# FP64 variant with FMA contraction (the flow's rounding floor); 64 layers
# end three times above it.
MIXED_WALL_LAYERS = 80


def make_workload(name: str, seed_offset: int = 0):
    from hydraphase import cases
    if name.startswith("cylinder"):
        nr, nt, nz = {"cylinder": (160, 256, 20), "cylinder_small": (40, 64, 16),
                      "cylinder_medium": (80, 128, 16)}.get(name, (0, 0, 0))
        if nr == 0:
            raise SystemExit(f"unknown workload {name}")
        spec = cases.cylinder(nr=nr, nt=nt, nz=nz, seed=1 + seed_offset, alpha_w_drop=1e-5, alpha_w_bg=1e-6)
        spec.flow["cfl"] = CYL_CFL
        return spec
    if name == "shock_bubble":
        # the small plain-method config: 20^3 hexes (48,000 tets), inviscid,
        # K = 5, SSP-RK3; air fraction 0.9/0.1 and CFL 0.05, the settings at
        # which these shock-bubble cases stay finite (CFL 0.4 blows up within
        # 25-100 steps in FP64 too)
        spec = cases.shock_bubble(n=20, alpha_min=0.1, seed=seed_offset)
        spec.flow["cfl"] = 0.05
        return spec
    raise SystemExit(f"unknown workload {name}")


def workload_config(spec, name):
    m = spec.mesh
    return {"workload": name, "cells": m.neles, "boundary_ghosts": m.nghosts,
            "rk_stages_per_step": 3 if spec.extra.get("rk_scheme", 0) == 1 else 4,
            "scheme": "SSP-RK3" if spec.extra.get("rk_scheme", 0) == 1 else "ESSPRK-4",
            "flux": "HLLC-Batten", "limiter_K": spec.extra.get("venkat_k", 0.3),
            "viscous": not spec.extra.get("inviscid", 0), "cfl": spec.flow["cfl"],
            "l2_policy": l2_policy(spec)}


def l2_policy(spec) -> str:
    gb = resident_gb(spec)
    if gb * 1e9 > 126e6:
        return f"state larger than L2 ({gb:.1f} GB resident per replica, L2 126 MB)"
    return f"state fits in L2 ({gb * 1e3:.0f} MB resident, L2 126 MB): L2-resident timings"


def resident_gb(spec) -> float:
    """Device bytes of one Case of this workload (FP64 parity variant)."""
    from hydraphase import PREC_FP64_PARITY
    from hydraphase.engine import estimate_bytes
    return estimate_bytes(spec.mesh, spec.params(precision=PREC_FP64_PARITY)) / 1e9


def dist_setup(backend: str):
    """Process group of a torchrun launch (None for one process).  The
    reference arm uses gloo (no device data crosses ranks); the CUDA arm
    uses nccl unless BENCH_BACKEND says otherwise."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier_max(pg, value: float, device) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier_sum(pg, value: float, device) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def alpha_g(cu: np.ndarray, flow: dict) -> np.ndarray:
    """alpha_g of a conserved state through the reference's pressure-
    equilibrium recovery (src/sr_primitive.F90:53-91)."""
    gg, gp, pinf = flow["gamag"], flow["gamap"], flow["pinf"]
    eg = cu[4] / cu[0] - 0.5 * (cu[1] ** 2 + cu[2] ** 2 + cu[3] ** 2) / cu[0] ** 2
    ep = cu[9] / cu[5] - 0.5 * (cu[6] ** 2 + cu[7] ** 2 + cu[8] ** 2) / cu[5] ** 2
    bbb = pinf * gp - cu[0] * (gg - 1) * eg - cu[5] * (gp - 1) * ep
    ccc = cu[0] * (gg - 1) * eg * pinf * gp
    pg = (-bbb + np.sqrt(bbb * bbb + 4 * ccc)) * 0.5
    return cu[0] * (gg - 1) * eg / pg


def accuracy(cu: np.ndarray, ref: np.ndarray, flow: dict) -> dict:
    """Relative L2 distances of a state to a reference state: mixture
    density, air volume fraction, and the largest over the ten conserved
    variables of each phase."""
    def rl2(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    per_var = [rl2(cu[k], ref[k]) for k in range(10)]
    return {"density": rl2(cu[0] + cu[5], ref[0] + ref[5]),
            "alpha_g": rl2(alpha_g(cu, flow), alpha_g(ref, flow)),
            "air_vars_max": max(per_var[:5]), "water_vars_max": max(per_var[5:])}


def profiled_traffic_per_cell(kernel: str):
    """DRAM bytes per cell of one launch of `kernel`, from the committed ncu
    summary of that kernel (profiles/<kernel>_*.md, line
    'dram_bytes_per_cell: X'), or None."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", kernel + "_*.md"))):
        m = re.search(r"dram_bytes_per_cell:\s*([0-9.]+)", open(path).read())
        if m:
            return float(m.group(1)), os.path.basename(path)
    return None


def profiled_pipes(kernel: str):
    """FP64-pipe and issue activity (fractions of peak over active cycles) of
    `kernel` from its committed ncu summary (lines 'fp64_pipe_active: X' and
    'issue_active: Y', percent), or None: what bounds a kernel that is not
    DRAM-bound."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", kernel + "_*.md"))):
        t = open(path).read()
        a = re.search(r"fp64_pipe_active:\s*([0-9.]+)", t)
        b = re.search(r"issue_active:\s*([0-9.]+)", t)
        if a and b:
            return {"fp64_pipe_active": float(a.group(1)) / 100, "issue_active": float(b.group(1)) / 100,
                    "source": "profiles/" + os.path.basename(path)}
    return None


def cpu_oracle_run(spec, threads: int, warmup: int, steps: int | None = None,
                   seconds_target: float | None = None):
    """The CPU restatement of the reference (oracle/, FP64, OpenMP over cells
    on `threads` host threads) on the same workload as the GPU arm: `warmup`
    untimed whole steps, then either `steps` timed steps or whole steps until
    `seconds_target` seconds of stepping have passed.  Returns
    (cell-stage updates/s, steps timed, seconds)."""
    import oracle as O
    m = spec.mesh
    O.set_threads(threads)
    orc = O.Oracle(O.params_from_flow(spec.flow, **spec.extra), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    if warmup > 0:
        orc.run(warmup)
    stages = 3 if spec.extra.get("rk_scheme", 0) == 1 else 4
    n, t_used = 0, 0.0
    while (steps is not None and n < steps) or (steps is None and t_used < seconds_target):
        t0 = time.perf_counter()
        orc.run(1)
        t_used += time.perf_counter() - t0
        n += 1
    orc.close()
    return m.neles * stages * n / t_used, n, t_used


def cpu_baseline(spec, name: str, threads: int, seconds_target: float = 12.0):
    """cpu_baseline of the GPU arm's line: the oracle on the identical
    workload, one untimed step, then whole steps for about seconds_target."""
    v, n, t = cpu_oracle_run(spec, threads, 1, seconds_target=seconds_target)
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the timed workload itself ({name}, {spec.mesh.neles} cells): {n} whole steps after "
                      f"1 untimed, {t:.1f} s", "same_config": True}


def serving_measure(n_cases: int, steps: int, repeats: int = 3):
    """The batched serving stream (shock-bubble cases of log-uniform size
    6k-400k cells, Poisson arrivals at 40/s, SSP-RK3) served in real time in
    the mixed and the plain FP64 variant, after tuning the per-cell kernel
    block size for each mesh-size class present.  The mixed stream is served
    `repeats` times (its rate follows the host's set-up work, which runs on
    the CPU next to the device work): the line reports the median run and the
    range of the aggregate rate.  The FP64 stream is served once."""
    from hydraphase import PREC_FP64_PARITY, PREC_MIXED, cases, tune
    from hydraphase.serve import Server
    t0 = time.perf_counter()
    reqs = cases.serving_stream(n_cases=n_cases, steps=steps)
    gen_s = time.perf_counter() - t0
    out = {"workload": f"shock-bubble stream: {n_cases} cases, cells log-U[6000, 400000], Poisson 40/s, "
                       f"{steps} SSP-RK3 steps each, CFL 0.05, HBM budget 150 GiB; time-to-solution "
                       f"from arrival to the final state on the host; after an untimed 25-step warm-up of every case",
           "cells_total": int(sum(r.spec.mesh.neles for r in reqs)), "generation_s": round(gen_s, 2)}
    reports = {}
    for name, prec in (("mixed", PREC_MIXED), ("fp64", PREC_FP64_PARITY)):
        blocks, modes, smodes = {}, {}, {}
        for r in reqs:
            cls = tune.size_class(r.spec.mesh.neles)
            if cls not in blocks:
                blocks[cls] = tune.tune_block_size(r.spec, precision=prec, steps=4)[0]
                modes[cls] = tune.tune_face_mode(r.spec, precision=prec, block_size=blocks[cls], steps=4)[0]
                smodes[cls] = tune.tune_step_mode(r.spec, precision=prec, block_size=blocks[cls],
                                                  face_mode=modes[cls], steps=4)[0]
        server = Server(150 << 30, precision=prec, max_active=16, chunk=25, chunk_cell_steps=10_000_000,
                        batch_cells=200000, block_size=blocks, face_mode=modes, step_mode=smodes, keep_state=True)
        # warm-up (untimed): every case of the stream for 25 steps, all
        # arriving at once, so the measured run pays no first-use costs
        # (module loading, pool growth to the stream's peak, worker start-up)
        server.run([type(r)(r.rid, 0.0, 25, r.spec) for r in reqs], realtime=False)
        runs = [server.run(reqs) for _ in range(repeats if name == "mixed" else 1)]
        rates = [r.summary()["updates_per_s"] for r in runs]
        rep_ = runs[int(np.argsort(rates)[len(rates) // 2])]          # the median run
        reports[name] = rep_
        out[name] = {**rep_.summary(), "block_size": blocks, "face_mode": modes,
                     "step_mode": {k: ("fused" if v == 2 else "graph") for k, v in smodes.items()}, "runs": len(runs),
                     "updates_per_s_range": [min(rates), max(rates)]}
    out["speedup_mixed_vs_fp64"] = out["mixed"]["updates_per_s"] / out["fp64"]["updates_per_s"]
    # each served mixed result against the served FP64 result of the same case
    fp = {r.rid: r for r in reports["fp64"].results}
    err = []
    for r in reports["mixed"].results:
        f = fp.get(r.rid)
        if r.error is None and f is not None and f.error is None and r.cu is not None and f.cu is not None:
            rho_m, rho_f = r.cu[0] + r.cu[5], f.cu[0] + f.cu[5]
            err.append(float(np.linalg.norm(rho_m - rho_f) / np.linalg.norm(rho_f)))
    if err:
        out["mixed_vs_fp64_density_rel_l2"] = {"median": float(np.median(err)), "max": float(np.max(err)),
                                               "cases": len(err), "steps": steps}
    return out


def overset_measure(steps: int):
    """The overset cylinder (background 200x120x20 hexes on [-10,30]x[-12,12]
    x[0,4], O-grid component 96x256x20 to r = 3D, hole r < 1.2D, two fringe
    layers): device-timed steps of the FP64 parity and the mixed variant with
    the fringe interpolated from its donors after every RK stage."""
    from hydraphase import PREC_FP64_PARITY, PREC_MIXED, Case, cases
    from hydraphase.engine import MeshArrays, overset_build, overset_hole_cut
    t0 = time.perf_counter()
    ov = cases.overset_cylinder(alpha_w_drop=1e-5, alpha_w_bg=1e-6)
    ov.spec.flow["cfl"] = CYL_CFL
    m = ov.spec.mesh
    t1 = time.perf_counter()
    # the library's wall-surface hole cut (within 0.7D of the wall faces, or
    # inside them) on the unblanked mesh, host and device, against r < 1.2D
    el1 = m.elem.copy()
    el1[:, 8] = 1
    m1 = MeshArrays(m.x, m.y, m.z, el1, m.ghost)
    overset_hole_cut(m1, ov.block, 6, 0.7, device=True)          # first-use costs
    th0 = time.perf_counter()
    hc_h, _ = overset_hole_cut(m1, ov.block, 6, 0.7)
    th1 = time.perf_counter()
    hc_d, _ = overset_hole_cut(m1, ov.block, 6, 0.7, device=True)
    th2 = time.perf_counter()
    hole_cut = {"host_s": round(th1 - th0, 3), "gpu_s": round(th2 - th1, 3),
                "gpu_equal_host": bool(np.array_equal(hc_h, hc_d)),
                "cells_differing_from_radius_rule": int((hc_h != m.elem[:, 8]).sum())}
    t1 = time.perf_counter()
    ib, tab = overset_build(m, ov.block, ov.layers, ov.outer_type)
    t2 = time.perf_counter()
    ib_d, tab_d = overset_build(m, ov.block, ov.layers, ov.outer_type, device=True)
    t3 = time.perf_counter()
    same = bool(np.array_equal(ib, ib_d) and np.array_equal(tab.fringe, tab_d.fringe) and
                np.array_equal(tab.donor, tab_d.donor) and np.array_equal(tab.weight, tab_d.weight))
    el = m.elem.copy()
    el[:, 8] = ib
    mesh = MeshArrays(m.x, m.y, m.z, el, m.ghost)
    out = {"workload": "overset cylinder: background 200x120x20 + O-grid 96x256x20 hexes (6 tets each), "
                       "hole r < 1.2D, 2 fringe layers, SSP-RK3, viscous",
           "cells": m.neles, "holes": int((m.elem[:, 8] == 0).sum()), "fringe": int(tab.fringe.size),
           "donor_fallbacks": int(tab.nfallback), "table_build_s": round(t2 - t1, 2),
           "table_build_gpu_s": round(t3 - t2, 3), "gpu_tables_equal_host": same,
           "mesh_generation_s": round(th0 - t0, 2), "hole_cut": hole_cut}
    states = {}
    for name, prec in (("fp64", PREC_FP64_PARITY), ("mixed", PREC_MIXED)):
        with Case(mesh, ov.spec.params(precision=prec)) as c:
            c.set_state(0.0, ov.spec.cu, ov.spec.ghost_prims)
            c.set_overset(tab)
            c.step(3, diagnostics=False)
            ms = c.step_timed(steps)
            pr = c.profile(1)
            share = pr["ms"][pr["kinds"].index("overset")] / sum(pr["ms"])
            _, states[name], _ = c.state()
        out[name] = {"value": m.neles * 3 * steps / (ms / 1e3), "ms_per_step": ms / steps,
                     "overset_kernel_share": share}
    out["mixed_rel_l2_vs_fp64"] = accuracy(states["mixed"], states["fp64"], ov.spec.flow)
    out["unit"] = UNIT
    return out


def partition_measure(spec, nparts: int, steps: int, check_steps: int = 3) -> dict:
    """The workload split into nparts parts with two halo layers
    (hydraphase.partition), run on this one GPU as the cases of one batch
    coupled by hp_set_halo (one dt; halo cells copied from their owners after
    every RK stage): device-timed steps, the halo share of the cells, and
    whether check_steps steps reproduce the single-mesh FP64 parity run bit
    for bit."""
    from hydraphase import PREC_FP64_PARITY, Case
    from hydraphase.partition import PartitionedCase, partition_case
    t0 = time.perf_counter()
    P = partition_case(spec, nparts)
    t1 = time.perf_counter()
    local = sum(p.spec.mesh.neles for p in P.parts)
    prm = spec.params(precision=PREC_FP64_PARITY)
    with PartitionedCase(P, prm) as pc:
        pc.set_state(0.0, spec.cu, spec.ghost_prims)
        dp = pc.step(check_steps)
        _, cu_p, gp_p = pc.state()
        ms = pc.step_timed(steps)
    with Case(spec.mesh, prm) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        ds = c.step(check_steps)
        _, cu_s, gp_s = c.state()
    same = bool(np.array_equal(cu_p, cu_s) and np.array_equal(gp_p, gp_s) and
                all(np.array_equal(dp[k], ds[k]) for k in ("time", "dt", "velmag", "diff")))
    stages = 3 if spec.extra.get("rk_scheme", 0) == 1 else 4
    return {"parts": nparts, "layout": "one GPU, the parts as one coupled batch",
            "cells": spec.mesh.neles, "local_cells": local, "halo_frac": local / spec.mesh.neles - 1.0,
            "value": spec.mesh.neles * stages * steps / (ms / 1e3), "ms_per_step": ms / steps, "unit": UNIT,
            "partition_s": round(t1 - t0, 2), f"bit_exact_vs_single_mesh_{check_steps}_steps": same}


def stress_measure(steps: int) -> dict:
    """Config 5, the precision stress: a 60 x 60 x 90-hex box (1,944,000
    tets, jitter +-0.15h, seed 3), a 5e9 Pa water shock on a 5 x 5 lattice of
    air bubbles, run `steps` steps in FP64 (parity), mixed and all-FP32;
    each result's error against FP64 and its positivity violations
    (hydraphase.stress)."""
    from hydraphase import cases, stress
    spec = cases.shock_lattice()
    res = stress.run(spec, steps, chunk=max(steps // 4, 1))
    return {"workload": f"shock lattice: {spec.mesh.neles} cells, 5e9 Pa water shock on a 5x5 air-bubble lattice, "
                        f"air fraction 0.9/0.1, SSP-RK3, CFL {spec.flow['cfl']}, {steps} steps",
            "cells": spec.mesh.neles, "steps": steps, **res}


def accuracy_run(spec, steps: int, wall_layers: int = 0) -> dict:
    """The mixed variant (and, with wall_layers > 0, the mixed variant with
    that many FP64 wall layers) against the FP64 parity variant after
    `steps` steps from the same initial state, on the timed workload (rel L2
    of mixture density, alpha_g and the conserved variables), with the FP64
    FMA variant's distance as the rounding floor and the NaN cells of every
    final state."""
    from hydraphase import PREC_FP64, PREC_FP64_PARITY, PREC_MIXED, Case
    runs = [("fp64", PREC_FP64_PARITY, {}), ("fp64_fma", PREC_FP64, {}), ("mixed", PREC_MIXED, {})]
    if wall_layers > 0:
        runs.append(("mixed_wall", PREC_MIXED, {"wall_fp64_layers": wall_layers}))
    states = {}
    for name, prec, over in runs:
        with Case(spec.mesh, spec.params(precision=prec, **over)) as c:
            c.set_state(0.0, spec.cu, spec.ghost_prims)
            c.step(steps, diagnostics=False)
            _, states[name], _ = c.state()
    out = {"steps": steps, "rel_l2_vs_fp64": accuracy(states["mixed"], states["fp64"], spec.flow),
           "fma_floor_rel_l2_vs_fp64": accuracy(states["fp64_fma"], states["fp64"], spec.flow),
           "nan_cells": {k: int((~np.isfinite(v)).any(axis=0).sum()) for k, v in states.items()}}
    if wall_layers > 0:
        out["wall_layers"] = wall_layers
        out["mixed_wall_rel_l2_vs_fp64"] = accuracy(states["mixed_wall"], states["fp64"], spec.flow)
    return out


def output_measure(steps: int = 300) -> dict:
    """Restart + Tecplot output of the 983k-cell cylinder (mixed variant)
    written while `steps` steps run (hp_output_async), against the same
    output written with the steps stopped: wall-clock seconds and the
    fraction of the write time hidden behind the steps."""
    import shutil
    from hydraphase import PREC_MIXED, Case
    spec = make_workload("cylinder_medium")
    d = tempfile.mkdtemp(prefix="hp_out_")
    try:
        with Case(spec.mesh, spec.params(precision=PREC_MIXED)) as c:
            c.set_state(0.0, spec.cu, spec.ghost_prims)
            c.step(3, diagnostics=False)
            c.sync()
            t0 = time.perf_counter()
            c.step(steps, diagnostics=False)
            c.sync()
            t_steps = time.perf_counter() - t0
            t0 = time.perf_counter()
            c.output_wait(c.output_async(os.path.join(d, "r1.in"), os.path.join(d, "t1.dat"), mesh=spec.mesh))
            t_write = time.perf_counter() - t0
            t0 = time.perf_counter()
            tk = c.output_async(os.path.join(d, "r2.in"), os.path.join(d, "t2.dat"), mesh=spec.mesh)
            c.step(steps, diagnostics=False)
            c.sync()
            t_steps_during = time.perf_counter() - t0
            c.output_wait(tk)
            t_both = time.perf_counter() - t0
            size = os.path.getsize(os.path.join(d, "r2.in")) + os.path.getsize(os.path.join(d, "t2.dat"))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return {"workload": f"cylinder 983,040 cells, mixed, {steps} steps; one restart + Tecplot file ({size / 1e6:.0f} MB)",
            "steps_s": round(t_steps, 3), "write_stopped_s": round(t_write, 3),
            "steps_while_writing_s": round(t_steps_during, 3), "steps_and_write_overlapped_s": round(t_both, 3),
            "hidden_fraction": round((t_steps + t_write - t_both) / t_write, 3) if t_write > 0 else None}


def run_reference_arm(args, world, rank, pg):
    """The reference's algorithm on the host cores, on the GPU arm's
    workload and step counts: the FP64 CPU restatement in oracle/ (the
    Fortran reference cannot be built here), --warmup untimed steps, then
    --steps timed whole steps.  Rank 0 only."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    spec = make_workload(args.workload)
    v, n, t = cpu_oracle_run(spec, threads, args.warmup, steps=args.steps)
    res = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"the GPU arm's workload ({args.workload}, {spec.mesh.neles} cells): {n} whole steps "
                     f"after {args.warmup} untimed, {t:.1f} s", "same_config": True}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "impl": "reference", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(spec, args.workload), "parallelism": f"replicas x{world}",
                       "precision": "fp64 bit-parity (no FMA)"},
            "note": "CPU restatement of the reference (oracle/), all host threads, rank 0",
            "ms_per_step": t * 1e3 / n, "cpu_baseline": res,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def measure_variant(spec, precision, steps, warmup, pg, device, **over):
    """Device-timed steps of one precision variant; returns numbers and the
    final state (for accuracy comparison)."""
    from hydraphase import Case
    p = spec.params(precision=precision, **over)
    c = Case(spec.mesh, p)
    c.set_state(0.0, spec.cu, spec.ghost_prims)
    c.step(warmup, diagnostics=False)
    c.sync()
    if pg is not None:
        pg.barrier()
    ms = c.step_timed(steps)
    if pg is not None:
        pg.barrier()
    info = c.info()
    prof = c.profile(2)
    d = c.step(1)
    t, cu, _ = c.state()
    c.close()
    return ms, info, prof, cu, d


def run_ours(args, world, rank, local, pg):
    import torch
    from hydraphase import PREC_FP64_PARITY, PREC_MIXED, Case
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    spec = make_workload(args.workload, seed_offset=rank)
    m = spec.mesh
    stages = 3 if spec.extra.get("rk_scheme", 0) == 1 else 4
    cells = m.neles
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    # --- headline: plain FP64 (bit-parity) path, device-timed -------------
    clocks = ClockSampler(local)
    clocks.start()
    ms64, info, prof64, cu64, d64 = measure_variant(spec, PREC_FP64_PARITY, args.steps, args.warmup, pg, device)
    clk = clocks.stop()
    t_max = barrier_max(pg, ms64, device) / 1e3
    total_updates = barrier_sum(pg, float(cells * stages * args.steps), device)
    value = total_updates / t_max

    # --- mixed precision variant ----------------------------------------
    msmx, infomx, profmx, cumx, dmx = measure_variant(spec, PREC_MIXED, args.steps, args.warmup, pg, device)
    tmx = barrier_max(pg, msmx, device) / 1e3
    value_mx = barrier_sum(pg, float(cells * stages * args.steps), device) / tmx
    acc_mx = accuracy(cumx, cu64, spec.flow)
    # the same with the cells near the walls in FP64
    wl = args.mixed_wall_layers
    if wl > 0:
        msmw, infomw, _, cumw, _ = measure_variant(spec, PREC_MIXED, args.steps, args.warmup, pg, device,
                                                   wall_fp64_layers=wl)
        value_mw = barrier_sum(pg, float(cells * stages * args.steps), device) / (barrier_max(pg, msmw, device) / 1e3)

    # --- end to end through the public API with host buffers -------------
    # inputs and results in pinned host memory, as a caller that streams
    # cases through the engine would hold them
    from hydraphase import Case as _Case

    def pinned_like(a):
        b = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape)
        b[...] = a
        return b
    cu_host = pinned_like(np.ascontiguousarray(spec.cu, np.float64))
    gp_host = pinned_like(np.ascontiguousarray(spec.ghost_prims, np.float64))
    cu_res = pinned_like(np.zeros(10 * m.neles))
    gp_res = pinned_like(np.zeros(max(6 * m.nghosts, 1)))
    c = _Case(m, spec.params(precision=PREC_FP64_PARITY))
    c.set_state(0.0, cu_host, gp_host)
    c.step(args.warmup, diagnostics=False)
    c.sync()
    if pg is not None:
        pg.barrier()
    t0 = time.perf_counter()
    c.set_state(0.0, cu_host, gp_host)
    diag = c.step(args.steps, diagnostics=True)
    _, cu_out, gp_out = c.state(out=(cu_res, gp_res))
    e2e_s = time.perf_counter() - t0
    c.close()
    e2e_max = barrier_max(pg, e2e_s, device)
    e2e_value = total_updates / e2e_max
    h2d = (cu_host.nbytes + gp_host.nbytes) / args.steps
    d2h = (cu_out.nbytes + gp_out.nbytes) / args.steps + 64

    # --- roofline of the dominant kernel (fused flux + source + update) ---
    kinds = prof64["kinds"]
    flux_ms = prof64["ms"][kinds.index("flux")] / max(prof64["launches"][kinds.index("flux")], 1)
    fb = flux_kernel_bytes(8, spec.extra.get("rk_scheme", 0))
    achieved = fb * cells / (flux_ms / 1e3) / 1e9
    step_ms = ms64 / args.steps
    achieved_step = STEP_BYTES_FP64 * cells * stages / (step_ms / 1e3) / 1e9
    share = {k: round(v / sum(prof64["ms"]), 4) for k, v in zip(kinds, prof64["ms"]) if v > 0}
    tp = profiled_traffic_per_cell("k_flux4")
    traffic = tp[0] * cells if tp else None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (O-grid cylinder generated in the reference's formats)",
        "config": {**workload_config(spec, args.workload), "parallelism": f"replicas x{world}",
                   "precision": "fp64 bit-parity (no FMA)"},
        "gpu_launches": int(info["kernels_per_step"]) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_flux (HLLC faces + sources + RK update)",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "peak_source": peak_src, "bytes_per_cell": fb, "traffic": traffic,
                     "traffic_source": (f"profiles/{tp[1]}: ncu dram bytes per cell x {cells} cells" if tp else None),
                     "pipes": profiled_pipes("k_flux4"),
                     "launch_ms": flux_ms,
                     "step_level": {"bytes_per_cell_stage": STEP_BYTES_FP64, "achieved": achieved_step,
                                    "frac": achieved_step / hbm_peak}},
        "kernel_share": share,
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "set_state (H2D from pinned host memory) + steps with per-step diagnostics + "
                        "get_state (D2H into pinned memory), wall clock"},
        "mixed": {"value": value_mx, "ms_per_step": msmx / args.steps, "speedup_vs_fp64": value_mx / value,
                  "rel_l2_vs_fp64_after_steps": acc_mx,
                  "dtype": "f32 fluxes/gradients, f64 state/EOS/reductions"},
        "nan_cells_after": float(d64["nan_cells"][0]),
    }
    if wl > 0:
        line["mixed_wall"] = {"wall_fp64_layers": wl, "value": value_mw, "ms_per_step": msmw / args.steps,
                              "speedup_vs_fp64": value_mw / value,
                              "rel_l2_vs_fp64_after_steps": accuracy(cumw, cu64, spec.flow),
                              "kernels_per_step": infomw["kernels_per_step"],
                              "dtype": "mixed; FP64 in the cells within wall_fp64_layers layers of the wall"}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(spec, args.workload, os.cpu_count() or 1)
    if world == 1 and rank == 0 and args.accuracy_steps > 0:
        line["mixed"]["accuracy"] = accuracy_run(spec, args.accuracy_steps, wl)
    if world == 1 and rank == 0 and not args.no_overset:
        line["overset"] = overset_measure(max(args.steps // 2, 5))
    if world == 1 and rank == 0 and args.partition_parts > 1:
        line["partitioned"] = partition_measure(spec, args.partition_parts, max(args.steps // 2, 5))
    if world == 1 and rank == 0 and not args.no_output:
        line["output"] = output_measure()
    if world == 1 and rank == 0 and args.stress_steps > 0:
        line["precision_stress"] = stress_measure(args.stress_steps)
    if world == 1 and rank == 0 and args.serving_cases > 0:
        sv = serving_measure(args.serving_cases, args.serving_steps)
        sv["mixed_served_vs_plain_fp64_value"] = sv["mixed"]["updates_per_s"] / value
        line["serving"] = sv
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_partitioned(args, world, rank, local, pg):
    """--partitioned: strong scaling of the workload over the ranks.  The
    mesh is split into one part per rank with two halo layers
    (hydraphase.partition); each rank steps its part in the FP64 parity
    variant, exchanging the halo after every RK stage and the dt minimum
    before every step through NCCL on the library's stream (DistComm; with
    one process, a single part and ThreadComm).  value = the whole mesh's
    cell-stage updates over the max-over-ranks device time."""
    import torch
    from hydraphase import PREC_FP64_PARITY
    from hydraphase.partition import DistComm, RankPart, ThreadComm, partition_case
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    spec = make_workload(args.workload)
    stages = 3 if spec.extra.get("rk_scheme", 0) == 1 else 4
    t0 = time.perf_counter()
    P = partition_case(spec, world)
    part_s = time.perf_counter() - t0
    comm = DistComm() if pg is not None else ThreadComm(1).bind(0)
    rp = RankPart(P, rank, spec.params(precision=PREC_FP64_PARITY), comm)
    cp, gp = P.scatter_state(spec.cu, spec.ghost_prims)[rank]
    rp.set_state(0.0, cp, gp)
    rp.step(args.warmup, diagnostics=False)
    rp.case.sync()
    if pg is not None:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ms = rp.case.step_timed(args.steps)
    clk = clocks.stop()
    if rp.error is not None:
        raise rp.error
    t_max = barrier_max(pg, ms, device) / 1e3
    local_cells = barrier_sum(pg, float(P.parts[rank].spec.mesh.neles), device)
    kernels = int(rp.case.info()["kernels_per_step"]) * args.steps
    rp.close()
    line = {
        "metric": METRIC, "value": spec.mesh.neles * stages * args.steps / t_max, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (O-grid cylinder generated in the reference's formats)",
        "config": {**workload_config(spec, args.workload),
                   "parallelism": f"partitioned x{world} (two-layer halo, exchange after every RK stage)",
                   "precision": "fp64 bit-parity (no FMA)", "halo_frac": local_cells / spec.mesh.neles - 1.0,
                   "partition_s": round(part_s, 2)},
        "gpu_launches": kernels, "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cylinder")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-cases", type=int, default=256,
                    help="cases of the serving stream measured after the step benchmark (0: skip)")
    ap.add_argument("--serving-steps", type=int, default=500)
    ap.add_argument("--no-overset", action="store_true", help="skip the overset cylinder measurement")
    ap.add_argument("--no-output", action="store_true", help="skip the asynchronous output measurement")
    ap.add_argument("--partition-parts", type=int, default=4,
                    help="parts of the partitioned-mesh measurement on this GPU (0 or 1: skip)")
    ap.add_argument("--partitioned", action="store_true",
                    help="strong scaling: one part of the workload mesh per rank, halo exchange over NCCL "
                         "(instead of one replica per rank)")
    ap.add_argument("--stress-steps", type=int, default=2000,
                    help="steps of the config-5 precision stress run in three precisions (0: skip)")
    ap.add_argument("--mixed-wall-layers", type=int, default=MIXED_WALL_LAYERS,
                    help="FP64 wall layers of the second mixed measurement (0: skip it)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 accuracy run on the timed workload (0: skip)")
    args = ap.parse_args()
    backend = "gloo" if args.impl == "reference" else os.environ.get("BENCH_BACKEND", "nccl")
    world, rank, local, pg = dist_setup(backend)
    try:
        if args.impl == "reference":
            rc = run_reference_arm(args, world, rank, pg)
        elif args.partitioned:
            rc = run_partitioned(args, world, rank, local, pg)
        else:
            rc = run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
