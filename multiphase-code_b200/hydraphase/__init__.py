"""B200-native residual-and-update engine for the two-phase six-equation
solver (reference: GauthamBijoy23/Multiphase-code, HydraPhase_60_FPC_5mill).

Host-side mirror of the C ABI in include/hydraphase.h; the kernels live in
libhydraphase.so next to this file (sm_100a).
"""
from ._lib import (HP_E_ARG, HP_E_CUDA, HP_E_IO, HP_E_NOMEM, HP_E_STATE, HP_E_UNSUPPORTED,
                   HydraError, PREC_FP32, PREC_FP64, PREC_FP64_PARITY, PREC_MIXED, LIB_PATH, lib)
from .engine import (Batch, Case, MeshArrays, make_params, read_flow, read_mesh, read_restart,
                     write_restart)

__all__ = ["Batch", "Case", "MeshArrays", "make_params", "read_flow", "read_mesh", "read_restart",
           "write_restart", "HydraError", "lib", "LIB_PATH", "PREC_FP64", "PREC_FP64_PARITY",
           "PREC_MIXED", "PREC_FP32", "HP_E_ARG", "HP_E_CUDA", "HP_E_IO", "HP_E_NOMEM", "HP_E_STATE",
           "HP_E_UNSUPPORTED"]
