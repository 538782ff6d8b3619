"""ctypes binding of libhydraphase.so (include/hydraphase.h).

The library is built in-tree (``make -C multiphase-code_b200``).  There is no
CPU fallback: if the shared library is missing, or no CUDA device is present
when a case is created, the calls fail with an exception.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# HYDRAPHASE_LIB selects another build of the same library (A/B timing).
LIB_PATH = os.environ.get("HYDRAPHASE_LIB", os.path.join(HERE, "libhydraphase.so"))

HP_OK, HP_E_ARG, HP_E_CUDA, HP_E_NOMEM, HP_E_IO, HP_E_STATE, HP_E_UNSUPPORTED = 0, -1, -2, -3, -4, -5, -6
PREC_FP64_PARITY, PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2, 3
HP_IBLANK_HALO1, HP_IBLANK_HALO2 = 2, 3      # partition halo layers
HP_X_DT, HP_X_HALO = 0, 1                    # exchange points (hp_set_exchange)
# hp_exchange_fn: (user, point, stream)
HP_EXCHANGE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p)

ERROR_NAMES = {HP_E_ARG: "HP_E_ARG", HP_E_CUDA: "HP_E_CUDA", HP_E_NOMEM: "HP_E_NOMEM",
               HP_E_IO: "HP_E_IO", HP_E_STATE: "HP_E_STATE", HP_E_UNSUPPORTED: "HP_E_UNSUPPORTED"}

_D = ctypes.c_double
_I = ctypes.c_int32
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int32)


class HpParams(ctypes.Structure):
    """hp_params: flow.in fields in file order plus the engine switches."""
    _fields_ = [(n, _D) for n in (
        "pmax", "pmin", "tgmax", "tgmin", "ugmax", "ugmin", "vgmax", "vgmin", "wgmax", "wgmin",
        "upmax", "upmin", "vpmax", "vpmin", "wpmax", "wpmin", "tpmax", "tpmin", "pinf", "gamap",
        "gamag", "cpp", "cpg", "amolg", "prg", "epslnmax", "epslnmin", "epslninf", "phipzero",
        "cfl")] + [
        ("niter", _I), ("itersub", _I), ("istart", _I), ("diap", _D), ("surfacetension", _D),
        ("myflux", _I), ("myorder", _I), ("as_", _D), ("ts", _D), ("face_mode", _I),
        ("venkat_k", _D), ("rk_scheme", _I), ("inviscid", _I), ("twall", _D), ("precision", _I),
        ("renumber", _I), ("block_size", _I), ("use_graph", _I), ("pad_", _D * 4),
        ("five_phase", _I)] + [(n, _D) for n in (
        "rhoq", "rhor", "rhos", "radq", "radr", "rads", "phiginit", "phipinit", "phiqinit", "phirinit",
        "phisinit")] + [("wall_fp64_layers", _I)]


class HpMesh(ctypes.Structure):
    _fields_ = [("nodes", _I), ("neles", _I), ("nghosts", _I), ("pghosts", _I),
                ("x", _DP), ("y", _DP), ("z", _DP), ("elem", _IP), ("ghost", _IP)]


class HpDiag(ctypes.Structure):
    _fields_ = [("time", _D), ("dt", _D), ("velmag", _D), ("diff", _D * 4), ("nan_cells", _D)]


class HpOverset(ctypes.Structure):
    _fields_ = [("nfringe", _I), ("fringe", ctypes.POINTER(_I)), ("donor", ctypes.POINTER(_I)),
                ("weight", _DP), ("nfallback", _I)]


class HydraError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the CUDA engine library; raise if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with 'make -C multiphase-code_b200'")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.hp_create.argtypes = [ctypes.POINTER(HpMesh), ctypes.POINTER(HpParams), ctypes.POINTER(vp)]
    L.hp_create_error.restype = ctypes.c_char_p
    L.hp_last_error.restype = ctypes.c_char_p
    L.hp_last_error.argtypes = [vp]
    L.hp_destroy.argtypes = [vp]
    L.hp_init_uniform.argtypes = [vp]
    L.hp_set_state.argtypes = [vp, _D, _DP, _DP]
    L.hp_step.argtypes = [vp, _I, ctypes.POINTER(HpDiag)]
    L.hp_sync.argtypes = [vp]
    L.hp_step_timed.argtypes = [vp, _I, _DP]
    L.hp_profile_steps.argtypes = [vp, _I, _DP, ctypes.POINTER(ctypes.c_int64), _I]
    L.hp_get_state.argtypes = [vp, _DP, _DP, _DP]
    L.hp_get_prims.argtypes = [vp, _DP]
    L.hp_device_state.argtypes = [vp, ctypes.POINTER(_DP), ctypes.POINTER(ctypes.c_int64)]
    L.hp_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                          ctypes.POINTER(ctypes.c_int64)]
    L.hp_create_batch.argtypes = [ctypes.POINTER(HpMesh), _I, ctypes.POINTER(HpParams), ctypes.POINTER(vp)]
    L.hp_case_count.argtypes = [vp, ctypes.POINTER(_I)]
    L.hp_set_state_case.argtypes = [vp, _I, _D, _DP, _DP]
    L.hp_get_state_case.argtypes = [vp, _I, _DP, _DP, _DP]
    L.hp_estimate_batch_bytes.argtypes = [ctypes.POINTER(HpMesh), _I, ctypes.POINTER(HpParams),
                                          ctypes.POINTER(ctypes.c_int64)]
    L.hp_overset_build.argtypes = [ctypes.POINTER(HpMesh), ctypes.POINTER(_I), _I, _I, ctypes.POINTER(_I),
                                   ctypes.POINTER(HpOverset)]
    L.hp_overset_build_gpu.argtypes = L.hp_overset_build.argtypes
    L.hp_overset_hole_cut.argtypes = [ctypes.POINTER(HpMesh), ctypes.POINTER(_I), _I, _D, ctypes.POINTER(_I),
                                      ctypes.POINTER(_I)]
    L.hp_overset_hole_cut_gpu.argtypes = L.hp_overset_hole_cut.argtypes
    L.hp_set_halo.argtypes = [vp, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                              ctypes.POINTER(_I)]
    L.hp_set_exchange.argtypes = [vp, HP_EXCHANGE_FN, vp]
    L.hp_set_halo_lists.argtypes = [vp, _I, ctypes.POINTER(_I), _I, ctypes.POINTER(_I)]
    L.hp_halo_pack.argtypes = [vp, vp]
    L.hp_halo_unpack.argtypes = [vp, vp]
    L.hp_dtmin_ptr.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64))]
    L.hp_free_overset.argtypes = [ctypes.POINTER(HpOverset)]
    L.hp_free_overset.restype = None
    L.hp_set_overset.argtypes = [vp, ctypes.POINTER(HpOverset)]
    L.hp_estimate_bytes.argtypes = [ctypes.POINTER(HpMesh), ctypes.POINTER(HpParams), ctypes.POINTER(ctypes.c_int64)]
    L.hp_poll.argtypes = [vp, ctypes.POINTER(_I)]
    L.hp_set_host_threads.argtypes = [_I]
    L.hp_dt_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, _I,
                                ctypes.POINTER(HpParams), ctypes.c_void_p, ctypes.c_void_p]
    L.hp_read_flow.argtypes = [ctypes.c_char_p, ctypes.POINTER(HpParams)]
    L.hp_read_mesh.argtypes = [ctypes.c_char_p, _I, ctypes.POINTER(HpMesh)]
    L.hp_free_mesh.argtypes = [ctypes.POINTER(HpMesh)]
    L.hp_read_restart.argtypes = [ctypes.c_char_p, _I, _I, _DP, _DP, _DP]
    L.hp_write_restart.argtypes = [ctypes.c_char_p, _I, _I, _D, _DP, _DP]
    L.hp_write_tecplot.argtypes = [ctypes.c_char_p, ctypes.POINTER(HpMesh), _DP]
    L.hp_output_async.argtypes = [vp, _I, ctypes.POINTER(HpMesh), ctypes.c_char_p, ctypes.c_char_p,
                                  ctypes.POINTER(_I)]
    L.hp_output_wait.argtypes = [vp, _I]
    for fn in ("hp_create", "hp_destroy", "hp_init_uniform", "hp_set_state", "hp_step", "hp_sync",
               "hp_step_timed", "hp_profile_steps", "hp_dt_noalloc", "hp_estimate_bytes", "hp_poll",
               "hp_create_batch", "hp_case_count", "hp_set_state_case", "hp_get_state_case",
               "hp_estimate_batch_bytes", "hp_overset_build", "hp_overset_build_gpu", "hp_set_overset",
               "hp_get_state", "hp_get_prims", "hp_device_state", "hp_info", "hp_read_flow",
               "hp_read_mesh", "hp_read_restart", "hp_write_restart", "hp_write_tecplot", "hp_output_async",
               "hp_output_wait", "hp_set_host_threads", "hp_overset_hole_cut", "hp_overset_hole_cut_gpu",
               "hp_set_halo", "hp_set_exchange", "hp_set_halo_lists", "hp_halo_pack", "hp_halo_unpack",
               "hp_dtmin_ptr"):
        getattr(L, fn).restype = ctypes.c_int
    _lib = L
    return L


KERNEL_KINDS = ("prim_start", "step_begin", "smooth1", "smooth2", "bc_visc", "visc", "prim_stage",
                "bc", "grad", "flux", "prim_end", "step_end", "serial", "overset", "halo", "qrs")

EXPORTED_SYMBOLS = (
    "hp_create", "hp_destroy", "hp_last_error", "hp_create_error", "hp_init_uniform",
    "hp_set_state", "hp_step", "hp_sync", "hp_step_timed", "hp_profile_steps", "hp_get_state", "hp_get_prims", "hp_device_state",
    "hp_info", "hp_read_flow", "hp_read_mesh", "hp_free_mesh", "hp_read_restart",
    "hp_write_restart", "hp_dt_noalloc", "hp_estimate_bytes", "hp_poll", "hp_create_batch", "hp_case_count",
    "hp_set_state_case", "hp_get_state_case", "hp_estimate_batch_bytes", "hp_overset_build", "hp_free_overset",
    "hp_set_overset", "hp_overset_build_gpu", "hp_write_tecplot", "hp_output_async", "hp_output_wait",
    "hp_set_host_threads", "hp_overset_hole_cut", "hp_overset_hole_cut_gpu", "hp_set_halo", "hp_set_exchange",
    "hp_set_halo_lists", "hp_halo_pack", "hp_halo_unpack", "hp_dtmin_ptr",
)
NOALLOC_MAX_CELLS = 1 << 24
