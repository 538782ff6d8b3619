"""hp_dt_noalloc: the time step computed without any device allocation.

Callers that cannot allocate device memory (a Fortran/OpenACC host whose
device arrays belong to its compiler runtime, or a framework whose pool owns
the GPU) pass their own buffers for the state, the cell sizes and the result;
the entry point's only scratch is a static device array.  These tests own the
buffers (allocated with torch, as such a caller's pool would) and call the
entry point through the C ABI:
  * twice in a row on two states whose time steps differ, each result equal
    to the dt that hp_step reports for the same state (bit-identical: both
    run the FP64 parity arithmetic);
  * on a state stored with a padded leading dimension (ld > ncells), as an
    OpenACC host may lay out its arrays;
  * on a smaller mesh right after a larger one, so the second call reads only
    the scratch slots it wrote itself.
The file is collected last so that a failure here stops a -x run only after
every other test has run.
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


def _noalloc_dt(spec, cu, pad=0):
    """dt through hp_dt_noalloc, the state stored column-major with `pad`
    unused cells after each column."""
    import torch
    n = spec.mesh.neles
    ld = n + pad
    host = np.full((10, ld), np.nan)            # padding is never read
    host[:, :n] = cu
    cn = torch.tensor(host, dtype=torch.float64, device="cuda")
    dl = torch.tensor(_cell_dl(spec), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    params = spec.params(precision=PREC_FP64_PARITY)
    rc = lib().hp_dt_noalloc(cn.data_ptr(), ld, dl.data_ptr(), n, ctypes.byref(params), out.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.item()


def test_dt_noalloc_matches_step_twice():
    spec = cases.cylinder(nr=6, nt=16, nz=2)
    second = spec.cu.copy()
    second[1:4] *= 1.7          # faster gas: a different, smaller time step
    second[6:9] *= 1.7
    got, ref = [], []
    for cu in (spec.cu, second):
        ref.append(_step_dt(spec, cu))
        got.append(_noalloc_dt(spec, cu))
        assert got[-1] == ref[-1]
    assert ref[0] != ref[1]     # the second comparison is a different answer


def test_dt_noalloc_padded_leading_dimension():
    spec = cases.cylinder(nr=6, nt=16, nz=2)
    assert _noalloc_dt(spec, spec.cu, pad=37) == _step_dt(spec, spec.cu)


def test_dt_noalloc_smaller_after_larger():
    big = cases.cylinder(nr=12, nt=32, nz=4)          # 9,216 cells: 36 scratch slots
    small = cases.shock_bubble(n=3, alpha_min=0.1)    # 162 cells: 1 slot
    assert big.mesh.neles > 16 * small.mesh.neles
    d_big = _noalloc_dt(big, big.cu)
    d_small = _noalloc_dt(small, small.cu)
    assert d_big == _step_dt(big, big.cu)
    assert d_small == _step_dt(small, small.cu)
    assert d_small != d_big


def test_dt_noalloc_rejects_oversize():
    import torch
    spec = cases.cylinder(nr=6, nt=16, nz=2)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    params = spec.params()
    rc = lib().hp_dt_noalloc(buf.data_ptr(), NOALLOC_MAX_CELLS + 1, buf.data_ptr(), NOALLOC_MAX_CELLS + 1,
                             ctypes.byref(params), buf.data_ptr(), None)
    assert rc == HP_E_ARG
