"""hp_dt_noalloc: the time step computed without any device allocation.

Callers that cannot allocate device memory (a Fortran/OpenACC host whose
device arrays belong to its compiler runtime, or a framework whose pool owns
the GPU) pass their own buffers for the state, the cell sizes and the result;
the entry point's only scratch is a static device array.  This test owns the
buffers (allocated with torch, as such a caller's pool would), calls the
entry point through the C ABI twice in a row on two different states, and
checks each result against the dt that hp_step reports for the same state
(bit-identical: both run the FP64 parity arithmetic).  It lives in a file
collected last so that a failure here stops a -x run only after every other
test has run.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from hydraphase import PREC_FP64_PARITY, Case, HP_E_ARG, cases, lib
from hydraphase._lib import NOALLOC_MAX_CELLS

pytestmark = pytest.mark.gpu


def _step_dt(spec, cu):
    """dt of the first step of `cu` through the handle-based entry point."""
    with Case(spec.mesh, spec.params(precision=PREC_FP64_PARITY)) as c:
        c.set_state(0.0, cu, spec.ghost_prims)
        return c.step(1)["dt"][0]


def _cell_dl(spec):
    m = spec.mesh
    orc = O.Oracle(O.params_from_flow(spec.flow, **spec.extra), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    return orc.geometry()[4, :m.neles].copy()


def test_dt_noalloc_matches_step_twice():
    import torch
    spec = cases.cylinder(nr=6, nt=16, nz=2)
    n = spec.mesh.neles
    dl = torch.tensor(_cell_dl(spec), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    params = spec.params(precision=PREC_FP64_PARITY)
    L = lib()
    second = spec.cu.copy()
    second[1:4] *= 1.7          # faster gas: a different, smaller time step
    second[6:9] *= 1.7
    for cu in (spec.cu, second):
        ref = _step_dt(spec, cu)
        cn = torch.tensor(np.ascontiguousarray(cu), dtype=torch.float64, device="cuda")
        rc = L.hp_dt_noalloc(cn.data_ptr(), n, dl.data_ptr(), n, ctypes.byref(params), out.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        assert out.item() == ref


def test_dt_noalloc_rejects_oversize():
    import torch
    spec = cases.cylinder(nr=6, nt=16, nz=2)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    params = spec.params()
    rc = lib().hp_dt_noalloc(buf.data_ptr(), NOALLOC_MAX_CELLS + 1, buf.data_ptr(), NOALLOC_MAX_CELLS + 1,
                             ctypes.byref(params), buf.data_ptr(), None)
    assert rc == HP_E_ARG
