"""Python mirror of the engine's C ABI: one ``Case`` per mesh on the GPU.

The method names follow the reference's time loop (src/main.F90:511-657):
``init_uniform`` is INIT_COND, ``set_state`` is the restart read,
``step`` runs main-loop iterations, ``state`` is what the restart writer
dumps.  Arrays use the reference's layout: conserved state column-major
(10, neles) in reference cell order, ghost primitives (6, nghosts) in
ghost-list order.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import (KERNEL_KINDS, HpDiag, HpMesh, HpOverset, HpParams, HydraError, PREC_FP64_PARITY, lib)

FLOW_FIELDS = (
    "pmax", "pmin", "tgmax", "tgmin", "ugmax", "ugmin", "vgmax", "vgmin", "wgmax", "wgmin",
    "upmax", "upmin", "vpmax", "vpmin", "wpmax", "wpmin", "tpmax", "tpmin", "pinf", "gamap",
    "gamag", "cpp", "cpg", "amolg", "prg", "epslnmax", "epslnmin", "epslninf", "phipzero", "cfl",
    "niter", "itersub", "istart", "diap", "surfacetension", "myflux", "myorder", "as_", "ts")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _check(rc: int, h=None):
    if rc != 0:
        L = lib()
        msg = (L.hp_last_error(h) if h else L.hp_create_error()) or b""
        raise HydraError(rc, msg.decode(errors="replace"))


def make_params(flow: dict | None = None, **over) -> HpParams:
    """hp_params from a flow.in dict (names as in the reference, ``as_`` for
    ``as``) plus engine switches (precision, renumber, use_graph, ...)."""
    p = HpParams()
    p.venkat_k = 0.3
    p.myflux = 2
    p.myorder = 2
    p.renumber = 1
    p.use_graph = 1
    p.precision = PREC_FP64_PARITY
    for src in (flow or {}), over:
        for k, v in src.items():
            if k == "as":
                k = "as_"
            setattr(p, k, v)
    return p


@dataclass
class MeshArrays:
    """Mesh in the reference's in-memory form (sr_geometry.F90:101-139)."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    elem: np.ndarray    # (neles, 9) int32: nod1..4, nc1..4, iblank
    ghost: np.ndarray   # (nghosts, 4) int32: nparent, nghost, ntype, nside

    @property
    def nodes(self):
        return int(self.x.shape[0])

    @property
    def neles(self):
        return int(self.elem.shape[0])

    @property
    def nghosts(self):
        return int(self.ghost.shape[0])


def _hp_mesh(mesh: MeshArrays, keep: list) -> HpMesh:
    arrs = [np.ascontiguousarray(mesh.x, np.float64), np.ascontiguousarray(mesh.y, np.float64),
            np.ascontiguousarray(mesh.z, np.float64), np.ascontiguousarray(mesh.elem, np.int32),
            np.ascontiguousarray(mesh.ghost, np.int32)]
    keep.extend(arrs)
    x, y, z, el, gh = arrs
    return HpMesh(mesh.nodes, mesh.neles, mesh.nghosts, 0, _dp(x), _dp(y), _dp(z), _ip(el), _ip(gh))


@dataclass
class OversetTable:
    """Fringe cells (1-based element ids), their four donors and barycentric
    weights, as hp_overset_build returns them."""
    fringe: np.ndarray      # (nf,) int32
    donor: np.ndarray       # (nf, 4) int32
    weight: np.ndarray      # (nf, 4) float64
    nfallback: int


def overset_build(mesh: MeshArrays, block, layers: int = 2, outer_type: int = 7, device: bool = False):
    """Fringe and donor tables of a two-block overset mesh (block[e] = 0
    background, 1 component; holes as iblank 0).  Returns (iblank, table):
    iblank marks the fringe with -1 and goes into the mesh given to Case.
    device=True runs the donor search on the current CUDA device
    (hp_overset_build_gpu); the tables are the same."""
    keep = []
    hm = _hp_mesh(mesh, keep)
    bl = np.ascontiguousarray(block, np.int32)
    ib = np.zeros(mesh.neles, np.int32)
    ov = HpOverset()
    build = lib().hp_overset_build_gpu if device else lib().hp_overset_build
    _check(build(ctypes.byref(hm), _ip(bl), int(layers), int(outer_type), _ip(ib), ctypes.byref(ov)))
    try:
        n = ov.nfringe
        fr = np.ctypeslib.as_array(ov.fringe, (n,)).copy() if n else np.zeros(0, np.int32)
        dn = np.ctypeslib.as_array(ov.donor, (n * 4,)).reshape(n, 4).copy() if n else np.zeros((0, 4), np.int32)
        w = np.ctypeslib.as_array(ov.weight, (n * 4,)).reshape(n, 4).copy() if n else np.zeros((0, 4))
        return ib, OversetTable(fr, dn, w, int(ov.nfallback))
    finally:
        lib().hp_free_overset(ctypes.byref(ov))


def overset_hole_cut(mesh: MeshArrays, block, wall_type: int = 6, margin: float = 0.0, device: bool = False):
    """Hole cut of a two-block overset mesh (hp_overset_hole_cut): background
    field cells within `margin` of, or enclosed by, the wall surface of the
    component block (its faces on ghosts of type wall_type) get iblank 0.
    Returns (iblank, nholes); put iblank into the mesh given to
    overset_build.  device=True tests the cells on the current CUDA device
    (hp_overset_hole_cut_gpu); the result is the same."""
    keep = []
    hm = _hp_mesh(mesh, keep)
    bl = np.ascontiguousarray(block, np.int32)
    ib = np.zeros(mesh.neles, np.int32)
    nh = ctypes.c_int32()
    cut = lib().hp_overset_hole_cut_gpu if device else lib().hp_overset_hole_cut
    _check(cut(ctypes.byref(hm), _ip(bl), int(wall_type), float(margin), _ip(ib), ctypes.byref(nh)))
    return ib, nh.value


def write_tecplot(path: str, mesh: MeshArrays, fields: np.ndarray):
    """The reference's Tecplot file (hp_write_tecplot) from the 13
    cell-centred fields (13, neles)."""
    keep = []
    hm = _hp_mesh(mesh, keep)
    f = np.ascontiguousarray(fields, np.float64)
    _check(lib().hp_write_tecplot(path.encode(), ctypes.byref(hm), _dp(f)))


def estimate_batch_bytes(meshes, params: HpParams) -> int:
    """Device bytes a Batch of these meshes would hold."""
    arr = (HpMesh * len(meshes))(*[HpMesh(m.nodes, m.neles, m.nghosts, 0, None, None, None, None, None)
                                   for m in meshes])
    b = ctypes.c_int64()
    _check(lib().hp_estimate_batch_bytes(arr, len(meshes), ctypes.byref(params), ctypes.byref(b)))
    return int(b.value)


def estimate_bytes(mesh: MeshArrays, params: HpParams) -> int:
    """Device bytes a Case of this mesh and precision would hold."""
    hm = HpMesh(mesh.nodes, mesh.neles, mesh.nghosts, 0, None, None, None, None, None)
    b = ctypes.c_int64()
    _check(lib().hp_estimate_bytes(ctypes.byref(hm), ctypes.byref(params), ctypes.byref(b)))
    return int(b.value)


class Case:
    """One mesh + solution resident on the current CUDA device."""

    def __init__(self, mesh: MeshArrays, params: HpParams):
        self.L = lib()
        self.mesh = mesh
        self.params = params
        self._keep = [np.ascontiguousarray(mesh.x, np.float64), np.ascontiguousarray(mesh.y, np.float64),
                      np.ascontiguousarray(mesh.z, np.float64), np.ascontiguousarray(mesh.elem, np.int32),
                      np.ascontiguousarray(mesh.ghost, np.int32)]
        x, y, z, el, gh = self._keep
        hm = HpMesh(mesh.nodes, mesh.neles, mesh.nghosts, 0, _dp(x), _dp(y), _dp(z), _ip(el), _ip(gh))
        h = ctypes.c_void_p()
        _check(self.L.hp_create(ctypes.byref(hm), ctypes.byref(params), ctypes.byref(h)))
        self.h = h
        self.neles = mesh.neles
        self.nghosts = mesh.nghosts
        self.neq = 22 if params.five_phase else 10

    def close(self):
        if getattr(self, "h", None):
            self.L.hp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_uniform(self):
        _check(self.L.hp_init_uniform(self.h), self.h)

    def set_state(self, time: float, cu: np.ndarray, ghost_prims: np.ndarray | None = None):
        cu = np.ascontiguousarray(cu, np.float64).reshape(-1)
        if cu.size != self.neq * self.neles:
            raise ValueError(f"cu must hold {self.neq} x neles values")
        gp = None if ghost_prims is None else np.ascontiguousarray(ghost_prims, np.float64).reshape(-1)
        _check(self.L.hp_set_state(self.h, float(time), _dp(cu), _dp(gp)), self.h)

    def step(self, nsteps: int, diagnostics: bool = True):
        """Run nsteps; returns a dict of per-step arrays (or None)."""
        if not diagnostics:
            _check(self.L.hp_step(self.h, int(nsteps), None), self.h)
            return None
        d = (HpDiag * max(int(nsteps), 1))()
        _check(self.L.hp_step(self.h, int(nsteps), d), self.h)
        arr = np.frombuffer(d, dtype=np.float64).reshape(-1, 8)[:nsteps]
        return {"time": arr[:, 0].copy(), "dt": arr[:, 1].copy(), "velmag": arr[:, 2].copy(),
                "diff": arr[:, 3:7].copy(), "nan_cells": arr[:, 7].copy()}

    def sync(self):
        _check(self.L.hp_sync(self.h), self.h)

    def set_overset(self, table: "OversetTable"):
        """Interpolate the fringe cells from their donors after every RK stage."""
        fr = np.ascontiguousarray(table.fringe, np.int32)
        dn = np.ascontiguousarray(table.donor, np.int32).reshape(-1)
        w = np.ascontiguousarray(table.weight, np.float64).reshape(-1)
        ov = HpOverset(int(fr.size), _ip(fr), _ip(dn), _dp(w), int(table.nfallback))
        _check(self.L.hp_set_overset(self.h, ctypes.byref(ov)), self.h)

    def poll(self) -> bool:
        """True while steps queued on this case's stream are still running."""
        busy = ctypes.c_int32()
        _check(self.L.hp_poll(self.h, ctypes.byref(busy)), self.h)
        return bool(busy.value)

    def step_timed(self, nsteps: int) -> float:
        """Run nsteps; device milliseconds from CUDA events on the case's stream."""
        ms = ctypes.c_double()
        _check(self.L.hp_step_timed(self.h, int(nsteps), ctypes.byref(ms)), self.h)
        return ms.value

    def profile(self, nsteps: int) -> dict:
        """Per-kernel-kind device time of nsteps launched eagerly with events."""
        n = len(KERNEL_KINDS)
        ms = np.zeros(n)
        cnt = np.zeros(n, np.int64)
        _check(self.L.hp_profile_steps(self.h, int(nsteps), _dp(ms),
                                       cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n), self.h)
        return {"kinds": list(KERNEL_KINDS), "ms": ms.tolist(), "launches": cnt.tolist()}

    def state(self, out=None):
        """(time, cu (neq, neles), ghost primitives (6, nghosts)); neq is 10,
        or 22 with the five-phase model.  out = (cu, gp): caller buffers
        (C-contiguous float64 of neq * neles and at least 6 * nghosts values,
        e.g. pinned memory) to fill instead."""
        t = ctypes.c_double()
        if out is None:
            cu = np.zeros(self.neq * self.neles)
            gp = np.zeros(6 * max(self.nghosts, 1))
        else:
            cu, gp = out
            if (cu.dtype != np.float64 or gp.dtype != np.float64 or not cu.flags.c_contiguous
                    or not gp.flags.c_contiguous or cu.size != self.neq * self.neles or gp.size < 6 * self.nghosts):
                raise ValueError("out must be C-contiguous float64 buffers of neq*neles and 6*nghosts values")
        _check(self.L.hp_get_state(self.h, ctypes.byref(t), _dp(cu), _dp(gp)), self.h)
        return t.value, cu.reshape(self.neq, self.neles), gp.reshape(-1)[:6 * self.nghosts].reshape(6, self.nghosts)

    def output_async(self, restart_path=None, tecplot_path=None, mesh: MeshArrays | None = None) -> int:
        """Start writing the current state (after the steps enqueued so far)
        to a restart file and/or a Tecplot file while later steps run
        (hp_output_async); returns a ticket for output_wait.  Tecplot needs
        the case's mesh, kept alive here until the wait."""
        keep = []
        hm = _hp_mesh(mesh, keep) if mesh is not None else None
        t = ctypes.c_int32()
        _check(self.L.hp_output_async(self.h, 0, ctypes.byref(hm) if hm is not None else None,
                                      restart_path.encode() if restart_path else None,
                                      tecplot_path.encode() if tecplot_path else None, ctypes.byref(t)), self.h)
        self._out_keep = getattr(self, "_out_keep", {})
        self._out_keep[t.value] = (keep, hm)
        return t.value

    def output_wait(self, ticket: int):
        """Block until the files of an output_async request are written."""
        try:
            _check(self.L.hp_output_wait(self.h, int(ticket)), self.h)
        finally:
            getattr(self, "_out_keep", {}).pop(int(ticket), None)

    def prims(self):
        out = np.zeros(14 * self.neles)
        _check(self.L.hp_get_prims(self.h, _dp(out)), self.h)
        return out.reshape(14, self.neles)

    def info(self):
        k, b, a = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(self.L.hp_info(self.h, ctypes.byref(k), ctypes.byref(b), ctypes.byref(a)), self.h)
        return {"kernels_per_step": k.value, "device_bytes": b.value, "aliased": bool(a.value)}


# --- reference file formats through the C ABI --------------------------------
def read_flow(path: str) -> HpParams:
    p = HpParams()
    _check(lib().hp_read_flow(path.encode(), ctypes.byref(p)))
    return p


def read_mesh(case_dir: str, rank: int = 0) -> MeshArrays:
    L = lib()
    m = HpMesh()
    _check(L.hp_read_mesh(case_dir.encode(), rank, ctypes.byref(m)))
    try:
        if m.pghosts:
            raise HydraError(-6, "proc_bc partition ghosts are not read: partition the whole mesh with "
                                 "hydraphase.partition instead")
        x = np.ctypeslib.as_array(m.x, (m.nodes,)).copy()
        y = np.ctypeslib.as_array(m.y, (m.nodes,)).copy()
        z = np.ctypeslib.as_array(m.z, (m.nodes,)).copy()
        el = np.ctypeslib.as_array(m.elem, (m.neles * 9,)).reshape(m.neles, 9).copy()
        gh = (np.ctypeslib.as_array(m.ghost, (m.nghosts * 4,)).reshape(m.nghosts, 4).copy()
              if m.nghosts else np.zeros((0, 4), np.int32))
    finally:
        L.hp_free_mesh(ctypes.byref(m))
    return MeshArrays(x, y, z, el, gh)


def read_restart(path: str, neles: int, nghosts: int):
    t = ctypes.c_double()
    cu = np.zeros(10 * neles)
    gp = np.zeros(6 * max(nghosts, 1))
    _check(lib().hp_read_restart(path.encode(), neles, nghosts, ctypes.byref(t), _dp(cu), _dp(gp)))
    return t.value, cu.reshape(10, neles), gp[:6 * nghosts].reshape(6, nghosts)


def write_restart(path: str, time: float, cu: np.ndarray, ghost_prims: np.ndarray):
    cu = np.ascontiguousarray(cu, np.float64)
    gp = np.ascontiguousarray(ghost_prims, np.float64)
    neles = cu.size // 10
    nghosts = gp.size // 6
    _check(lib().hp_write_restart(path.encode(), neles, nghosts, float(time), _dp(cu), _dp(gp)))


class Batch:
    """Several cases (same parameters) in one handle: their cell and ghost
    lists are concatenated on the device and every kernel of a step sweeps
    all of them in one launch (hp_create_batch).  Each case keeps its own
    dt, time and diagnostics; its results are those it would have alone."""

    def __init__(self, meshes, params: HpParams):
        self.L = lib()
        self.params = params
        self._keep = []
        arr = (HpMesh * len(meshes))(*[_hp_mesh(m, self._keep) for m in meshes])
        h = ctypes.c_void_p()
        _check(self.L.hp_create_batch(arr, len(meshes), ctypes.byref(params), ctypes.byref(h)))
        self.h = h
        self.neles = [m.neles for m in meshes]
        self.neq = 22 if params.five_phase else 10
        self.nghosts = [m.nghosts for m in meshes]

    @property
    def ncase(self) -> int:
        return len(self.neles)

    def close(self):
        if getattr(self, "h", None):
            self.L.hp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, c: int, time: float, cu: np.ndarray, ghost_prims: np.ndarray | None = None):
        cu = np.ascontiguousarray(cu, np.float64).reshape(-1)
        if cu.size != self.neq * self.neles[c]:
            raise ValueError("cu must hold %d x neles values of case %d" % (self.neq, c))
        gp = None if ghost_prims is None else np.ascontiguousarray(ghost_prims, np.float64).reshape(-1)
        _check(self.L.hp_set_state_case(self.h, int(c), float(time), _dp(cu), _dp(gp)), self.h)

    def step(self, nsteps: int, diagnostics: bool = True):
        """Run nsteps on every case; per-case lists of per-step arrays."""
        if not diagnostics:
            _check(self.L.hp_step(self.h, int(nsteps), None), self.h)
            return None
        d = (HpDiag * max(int(nsteps) * self.ncase, 1))()
        _check(self.L.hp_step(self.h, int(nsteps), d), self.h)
        arr = np.frombuffer(d, dtype=np.float64).reshape(-1, 8)[:nsteps * self.ncase].reshape(self.ncase, nsteps, 8)
        return [{"time": a[:, 0].copy(), "dt": a[:, 1].copy(), "velmag": a[:, 2].copy(),
                 "diff": a[:, 3:7].copy(), "nan_cells": a[:, 7].copy()} for a in arr]

    def sync(self):
        _check(self.L.hp_sync(self.h), self.h)

    def poll(self) -> bool:
        busy = ctypes.c_int32()
        _check(self.L.hp_poll(self.h, ctypes.byref(busy)), self.h)
        return bool(busy.value)

    def step_timed(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        _check(self.L.hp_step_timed(self.h, int(nsteps), ctypes.byref(ms)), self.h)
        return ms.value

    def state(self, c: int):
        t = ctypes.c_double()
        ne, ng = self.neles[c], self.nghosts[c]
        cu = np.zeros(self.neq * ne)
        gp = np.zeros(6 * max(ng, 1))
        _check(self.L.hp_get_state_case(self.h, int(c), ctypes.byref(t), _dp(cu), _dp(gp)), self.h)
        return t.value, cu.reshape(self.neq, ne), gp[:6 * ng].reshape(6, ng)
