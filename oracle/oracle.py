"""ctypes binding of the CPU oracle plus readers for the reference's input and
restart files.

TEST INFRASTRUCTURE ONLY: this module is the checker used by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs.  The product
library (multiphase-code_b200/) never imports it.

File formats follow the reference (paths relative to HydraPhase_60_FPC_5mill/):
  flow.in                 src/sr_Read_flow.F90:19-268 (one list-directed READ per
                          non-comment line, in a fixed order)
  grid_procNNNN.dat       src/sr_geometry.F90:101-128
  bc_procNNNN.in          src/sr_geometry.F90:131-134, src/main.F90:234-236
  proc_bcNNNN.in          src/sr_geometry.F90:136-139
  restartNNNN.in          src/main.F90:427-441 (read) and :812-828 (write)
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# flow.in groups in file order: (names, types)
FLOW_GROUPS = [
    (("pmax", "pmin"), (float, float)),
    (("tgmax", "tgmin"), (float, float)),
    (("ugmax", "ugmin"), (float, float)),
    (("vgmax", "vgmin"), (float, float)),
    (("wgmax", "wgmin"), (float, float)),
    (("upmax", "upmin"), (float, float)),
    (("vpmax", "vpmin"), (float, float)),
    (("wpmax", "wpmin"), (float, float)),
    (("tpmax", "tpmin"), (float, float)),
    (("pinf", "gamap"), (float, float)),
    (("gamag", "cpp"), (float, float)),
    (("cpg", "amolg"), (float, float)),
    (("prg", "epslnmax"), (float, float)),
    (("epslnmin", "epslninf", "phipzero"), (float, float, float)),
    (("cfl", "niter", "itersub"), (float, int, int)),
    (("istart", "diap"), (int, float)),
    (("surfacetension", "myflux"), (float, int)),
    (("myorder", "as_", "ts"), (int, float, float)),
]
# groups read only by the five-phase model; optional (the two-phase build
# stops reading after myorder, as, ts)
FLOW_GROUPS_OPT = [
    (("rhoq", "rhor", "rhos"), (float, float, float)),
    (("radq", "radr", "rads"), (float, float, float)),
    (("phiginit", "phipinit", "phiqinit", "phirinit", "phisinit"), (float,) * 5),
]


class OrParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "pmax", "pmin", "tgmax", "tgmin", "ugmax", "ugmin", "vgmax", "vgmin",
        "wgmax", "wgmin", "upmax", "upmin", "vpmax", "vpmin", "wpmax", "wpmin",
        "tpmax", "tpmin", "pinf", "gamap", "gamag", "cpp", "cpg", "amolg", "prg",
        "epslnmax", "epslnmin", "epslninf", "phipzero", "cfl")] + [
        ("niter", ctypes.c_int32), ("itersub", ctypes.c_int32),
        ("istart", ctypes.c_int32), ("diap", ctypes.c_double),
        ("surfacetension", ctypes.c_double), ("myflux", ctypes.c_int32),
        ("myorder", ctypes.c_int32), ("as_", ctypes.c_double), ("ts", ctypes.c_double),
        ("nan_mode", ctypes.c_int32), ("venkat_k", ctypes.c_double),
        ("rk_scheme", ctypes.c_int32), ("inviscid", ctypes.c_int32),
        ("twall", ctypes.c_double), ("pad_", ctypes.c_double * 3),
        ("five_phase", ctypes.c_int32), ("rhoq", ctypes.c_double), ("rhor", ctypes.c_double),
        ("rhos", ctypes.c_double), ("radq", ctypes.c_double), ("radr", ctypes.c_double),
        ("rads", ctypes.c_double), ("phiqinit", ctypes.c_double), ("phirinit", ctypes.c_double),
        ("phisinit", ctypes.c_double)]


def _fortran_value(tok: str, typ):
    tok = tok.strip()
    if typ is int:
        return int(tok)
    return float(tok.replace("d", "e").replace("D", "e"))


def parse_flow_in(text: str) -> dict:
    """Restatement of src/sr_Read_flow.F90:19-268: each group consumes the
    next non-blank, non-'#' line whose list-directed read succeeds."""
    lines = text.splitlines()
    pos = 0
    out: dict = {}
    for names, types in FLOW_GROUPS + FLOW_GROUPS_OPT:
        while True:
            if pos >= len(lines):
                if (names, types) in FLOW_GROUPS_OPT:
                    return out
                raise ValueError(f"flow.in ended before {names}")
            line = lines[pos]
            pos += 1
            if not line.strip() or line[:1] == "#":
                continue
            if "#" in line:
                line = line[: line.index("#")]
            toks = line.replace(",", " ").split()
            if len(toks) < len(names):
                continue
            try:
                vals = [_fortran_value(t, ty) for t, ty in zip(toks, types)]
            except ValueError:
                continue
            out.update(zip(names, vals))
            break
    return out


def default_params(**over) -> OrParams:
    p = OrParams()
    p.venkat_k = 0.3
    for k, v in over.items():
        setattr(p, k, v)
    return p


def params_from_flow(flow: dict, **over) -> OrParams:
    p = default_params()
    for k, v in flow.items():
        setattr(p, k, v)
    for k, v in over.items():
        setattr(p, k, v)
    return p


@dataclass
class Mesh:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    elem: np.ndarray        # (neles, 9) int32: nod1..4, nc1..4, iblank
    ghost: np.ndarray       # (nghosts, 4) int32: nparent, nghost, ntype, nside
    gid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    @property
    def nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def neles(self) -> int:
        return int(self.elem.shape[0])

    @property
    def nghosts(self) -> int:
        return int(self.ghost.shape[0])


def read_grid(path: str):
    import pandas as pd
    with open(path) as f:
        nodes, neles = (int(t) for t in f.readline().split()[:2])
    nd = pd.read_csv(path, sep=r"\s+", header=None, skiprows=1, nrows=nodes,
                     usecols=[0, 1, 2, 3, 4], engine="c", float_precision="round_trip").to_numpy()
    el = pd.read_csv(path, sep=r"\s+", header=None, skiprows=1 + nodes, nrows=neles,
                     usecols=list(range(10)), engine="c").to_numpy(dtype=np.int64)
    order = nd[:, 0].astype(np.int64) - 1
    x = np.zeros(nodes); y = np.zeros(nodes); z = np.zeros(nodes)
    gid = np.zeros(nodes, np.int32)
    x[order] = nd[:, 1]; y[order] = nd[:, 2]; z[order] = nd[:, 3]
    gid[order] = nd[:, 4].astype(np.int32)
    elem = np.zeros((neles, 9), np.int32)
    elem[el[:, 0] - 1] = el[:, 1:10]
    return x, y, z, gid, elem


def read_bc(path: str) -> np.ndarray:
    with open(path) as f:
        n = int(f.readline().split()[0])
        data = np.array(f.read().split()[: 4 * n], dtype=np.int64)
    return data.reshape(n, 4).astype(np.int32)


def read_case_dir(case_dir: str, rank: int = 0) -> tuple[dict, Mesh]:
    flow = parse_flow_in(open(os.path.join(case_dir, "flow.in")).read())
    g = os.path.join(case_dir, "geometry_files")
    x, y, z, gid, elem = read_grid(os.path.join(g, f"grid_proc{rank:04d}.dat"))
    ghost = read_bc(os.path.join(g, f"bc_proc{rank:04d}.in"))
    with open(os.path.join(g, f"proc_bc{rank:04d}.in")) as f:
        pgh = int(f.readline().split()[0])
    if pgh != 0:
        raise ValueError("partition ghosts are not supported (single partition)")
    return flow, Mesh(x, y, z, elem, ghost, gid)


def read_restart(path: str, neles: int, nghosts: int, neq: int = 10):
    """src/main.F90:431-438: time, cu(neles, neq) column-major, then ug, vg, wg,
    pg, tg, rog at the ghosts (list-directed; record boundaries are free)."""
    toks = open(path).read().split()
    need = 1 + neles * neq + 6 * nghosts
    if len(toks) < need:
        raise ValueError(f"restart file has {len(toks)} values, need {need}")
    vals = np.array(toks[:need], dtype=np.float64)
    t = float(vals[0])
    cu = vals[1:1 + neles * neq].copy()
    gp = vals[1 + neles * neq:].reshape(6, nghosts).copy()
    return t, cu, gp


def read_velocity_dat(path: str) -> np.ndarray:
    return np.loadtxt(path, dtype=np.float64).reshape(-1, 2)


def build() -> str:
    src = os.path.join(HERE, "hydra_oracle.c")
    if (not os.path.exists(LIB_PATH)
            or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        L = _lib
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.POINTER(OrParams), ctypes.c_int32, ctypes.c_int32,
                                ctypes.c_int32, dp, dp, dp, ip, ip]
        L.or_destroy.argtypes = [ctypes.c_void_p]
        L.or_init_uniform.argtypes = [ctypes.c_void_p]
        L.or_set_state.argtypes = [ctypes.c_void_p, ctypes.c_double, dp, dp]
        L.or_run.argtypes = [ctypes.c_void_p, ctypes.c_int32, dp, dp, dp]
        L.or_run.restype = ctypes.c_int
        L.or_time.restype = ctypes.c_double
        L.or_time.argtypes = [ctypes.c_void_p]
        L.or_last_dt.restype = ctypes.c_double
        L.or_last_dt.argtypes = [ctypes.c_void_p]
        L.or_ntot.restype = ctypes.c_int32
        L.or_ntot.argtypes = [ctypes.c_void_p]
        for fn in ("or_get_cu", "or_get_cn", "or_get_prims", "or_get_geometry",
                   "or_get_ghost_restart", "or_get_rhs", "or_get_d24", "or_get_vis",
                   "or_get_grad"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, dp]
        for fn in ("or_primitive", "or_primitiveplusbc", "or_derivative", "or_venkat",
                   "or_smooth", "or_viscous", "or_flux"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.or_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.or_set_threads.argtypes = [ctypes.c_int]
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.or_overset_build.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, dp, dp, dp, ip, ip, ip,
                                       ctypes.c_int32, ctypes.c_int32, ip, i32p, ip, ip, dp, i32p]
        L.or_overset_build.restype = ctypes.c_int
        L.or_set_overset.argtypes = [ctypes.c_void_p, ctypes.c_int32, ip, ip, dp]
        L.or_overset_hole_cut.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, dp, dp, dp, ip, ip,
                                          ip, ctypes.c_int32, ctypes.c_double, ip, i32p]
        L.or_overset_hole_cut.restype = ctypes.c_int
    return _lib


def set_threads(n: int) -> None:
    """Threads for the cell loops (meshes without aliased ghosts only)."""
    lib().or_set_threads(int(n))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def overset_build(mesh: Mesh, block, layers: int, outer_type: int):
    """Fringe cells, donors and weights of a two-block overset mesh, by the
    oracle's restatement of the rules; returns (iblank, fringe (1-based),
    donor (nf, 4), weight (nf, 4), nfallback)."""
    ne = mesh.neles
    keep = [np.ascontiguousarray(mesh.x, np.float64), np.ascontiguousarray(mesh.y, np.float64),
            np.ascontiguousarray(mesh.z, np.float64), np.ascontiguousarray(mesh.elem, np.int32),
            np.ascontiguousarray(mesh.ghost, np.int32), np.ascontiguousarray(block, np.int32)]
    ib = np.zeros(ne, np.int32)
    fr = np.zeros(ne, np.int32)
    dn = np.zeros(4 * ne, np.int32)
    w = np.zeros(4 * ne, np.float64)
    nf, nfb = ctypes.c_int32(), ctypes.c_int32()
    x, y, z, el, gh, bl = keep
    lib().or_overset_build(mesh.nodes, ne, mesh.nghosts, _dp(x), _dp(y), _dp(z), _ip(el), _ip(gh), _ip(bl),
                           int(layers), int(outer_type), _ip(ib), ctypes.byref(nf), _ip(fr), _ip(dn), _dp(w),
                           ctypes.byref(nfb))
    n = nf.value
    return ib, fr[:n].copy(), dn[:4 * n].reshape(n, 4).copy(), w[:4 * n].reshape(n, 4).copy(), nfb.value


def overset_hole_cut(mesh: Mesh, block, wall_type: int, margin: float):
    """Hole cut of a two-block overset mesh by the oracle's restatement of
    the rule: returns (iblank, nholes); background field cells within
    `margin` of, or enclosed by, the component's wall surface become 0."""
    keep = [np.ascontiguousarray(mesh.x, np.float64), np.ascontiguousarray(mesh.y, np.float64),
            np.ascontiguousarray(mesh.z, np.float64), np.ascontiguousarray(mesh.elem, np.int32),
            np.ascontiguousarray(mesh.ghost, np.int32), np.ascontiguousarray(block, np.int32)]
    x, y, z, el, gh, bl = keep
    ib = np.zeros(mesh.neles, np.int32)
    nh = ctypes.c_int32()
    rc = lib().or_overset_hole_cut(mesh.nodes, mesh.neles, mesh.nghosts, _dp(x), _dp(y), _dp(z), _ip(el), _ip(gh),
                                   _ip(bl), int(wall_type), float(margin), _ip(ib), ctypes.byref(nh))
    if rc != 0:
        raise ValueError("no wall face of the given type on the component block")
    return ib, nh.value


class Oracle:
    """One case held by the CPU oracle."""

    def __init__(self, params: OrParams, mesh: Mesh):
        self.L = lib()
        self.params = params
        self.mesh = mesh
        self._keep = [np.ascontiguousarray(mesh.x, np.float64),
                      np.ascontiguousarray(mesh.y, np.float64),
                      np.ascontiguousarray(mesh.z, np.float64),
                      np.ascontiguousarray(mesh.elem, np.int32),
                      np.ascontiguousarray(mesh.ghost, np.int32)]
        x, y, z, el, gh = self._keep
        self.h = self.L.or_create(ctypes.byref(params), mesh.nodes, mesh.neles,
                                  mesh.nghosts, _dp(x), _dp(y), _dp(z), _ip(el), _ip(gh))
        if not self.h:
            raise ValueError(f"myflux must be 1 (HLLC-Zien), 2 (HLLC-Batten) or 3 (Jameson), not {params.myflux}")
        self.neles = mesh.neles
        self.nghosts = mesh.nghosts
        self.ntot = mesh.neles + mesh.nghosts

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_uniform(self):
        self.L.or_init_uniform(self.h)

    @property
    def neq(self) -> int:
        return 22 if self.params.five_phase else 10

    def set_state(self, time: float, cu_elem: np.ndarray, ghost_prims=None):
        cu = np.ascontiguousarray(cu_elem, np.float64).ravel()
        assert cu.size == self.neq * self.neles
        gp = None if ghost_prims is None else np.ascontiguousarray(ghost_prims, np.float64).ravel()
        self.L.or_set_state(self.h, float(time), _dp(cu), _dp(gp) if gp is not None else None)

    def run(self, nsteps: int):
        t = np.zeros(nsteps); v = np.zeros(nsteps); d = np.zeros((nsteps, 4))
        self.L.or_run(self.h, nsteps, _dp(t), _dp(v), _dp(d))
        return t, v, d

    def _get(self, fn, shape):
        out = np.zeros(int(np.prod(shape)), np.float64)
        getattr(self.L, fn)(self.h, _dp(out))
        return out.reshape(shape)

    def cu(self):
        return self._get("or_get_cu", (self.neq, self.ntot))

    def cn(self):
        return self._get("or_get_cn", (self.neq, self.ntot))

    def prims(self):
        return self._get("or_get_prims", (16, self.ntot))

    def geometry(self):
        return self._get("or_get_geometry", (22, self.ntot))

    def ghost_restart(self):
        return self._get("or_get_ghost_restart", (6, self.nghosts))

    def rhs(self):
        return self._get("or_get_rhs", (self.neq, self.neles))

    def d24(self):
        return self._get("or_get_d24", (self.neq, self.neles))

    def vis(self):
        return self._get("or_get_vis", (8, self.neles))

    def grad(self):
        return self._get("or_get_grad", (40, self.ntot))

    @property
    def time(self) -> float:
        return self.L.or_time(self.h)

    @property
    def dt(self) -> float:
        return self.L.or_last_dt(self.h)

    def call(self, phase: str):
        getattr(self.L, "or_" + phase)(self.h)

    def set_dt(self, dt: float):
        self.L.or_set_dt(self.h, float(dt))

    def set_overset(self, fringe, donor, weight):
        """Fringe table applied after every RK stage (see overset_build)."""
        self._ov = [np.ascontiguousarray(fringe, np.int32), np.ascontiguousarray(donor, np.int32).ravel(),
                    np.ascontiguousarray(weight, np.float64).ravel()]
        f, d, w = self._ov
        self.L.or_set_overset(self.h, f.size, _ip(f), _ip(d), _dp(w))
