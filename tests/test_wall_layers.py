"""FP64 wall layers of the mixed variant (hp_params.wall_fp64_layers): the
cells within n breadth-first layers of a wall ghost take their viscous
terms, gradients, limiter, fluxes, sources and RK update from the FP64
kernels, the rest of the mesh stays FP32.

With every cell in the layers the step is the FP64 (FMA) variant's, bit for
bit.  On the viscous cylinder the mixed variant's distance to the reference
grows from the cells near the wall; the layers keep the mixed step within
1e-5 of the oracle where plain mixed drifts away.
"""
import os

import numpy as np
import pytest

import oracle as O
from hydraphase import PREC_FP64, PREC_MIXED, Case, cases


def _cylinder(nz):
    spec = cases.cylinder(nr=40, nt=64, nz=nz, alpha_w_drop=1e-5, alpha_w_bg=1e-6)
    spec.flow["cfl"] = 0.25
    return spec


def _run(spec, steps, **over):
    with Case(spec.mesh, spec.params(**over)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        d = c.step(steps)
        _, cu, _ = c.state()
        k = c.info()["kernels_per_step"]
    return cu, d, k


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _alpha_g(cu, flow):
    """alpha_g through the pressure-equilibrium recovery of
    src/sr_primitive.F90:53-91 (surface tension zero)."""
    gg, gp, pinf = flow["gamag"], flow["gamap"], flow["pinf"]
    eg = cu[4] / cu[0] - 0.5 * (cu[1] ** 2 + cu[2] ** 2 + cu[3] ** 2) / cu[0] ** 2
    ep = cu[9] / cu[5] - 0.5 * (cu[6] ** 2 + cu[7] ** 2 + cu[8] ** 2) / cu[5] ** 2
    bbb = pinf * gp - cu[0] * (gg - 1) * eg - cu[5] * (gp - 1) * ep
    ccc = cu[0] * (gg - 1) * eg * pinf * gp
    pg = (-bbb + np.sqrt(bbb * bbb + 4 * ccc)) * 0.5
    return cu[0] * (gg - 1) * eg / pg


@pytest.mark.gpu
def test_every_cell_in_the_layers_is_the_fp64_variant():
    spec = _cylinder(4)
    cu64, d64, k64 = _run(spec, 20, precision=PREC_FP64)
    cuw, dw, kw = _run(spec, 20, precision=PREC_MIXED, wall_fp64_layers=1 << 20)
    np.testing.assert_array_equal(cuw, cu64)
    np.testing.assert_array_equal(dw["dt"], d64["dt"])
    _, _, k0 = _run(spec, 1, precision=PREC_MIXED)
    assert kw == k0 + 1 + 3 * 2          # FP64 viscous once, gradients and fluxes per stage


@pytest.mark.gpu
def test_wall_layers_within_1e5_of_the_oracle_after_300_steps():
    spec = _cylinder(4)
    m = spec.mesh
    O.set_threads(os.cpu_count() or 1)
    orc = O.Oracle(O.params_from_flow(spec.flow, **spec.extra), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    orc.run(300)
    ref = orc.cu()[:, :m.neles]
    orc.close()
    rho_ref, ag_ref = ref[0] + ref[5], _alpha_g(ref, spec.flow)
    err = {}
    for name, over in (("mixed", {}), ("wall", {"wall_fp64_layers": 16})):
        cu, _, _ = _run(spec, 300, precision=PREC_MIXED, **over)
        assert np.isfinite(cu).all()
        err[name] = (_rel(cu[0] + cu[5], rho_ref), _rel(_alpha_g(cu, spec.flow), ag_ref))
    assert err["wall"][0] <= 1e-5 and err["wall"][1] <= 1e-5, err
    assert err["wall"][0] <= 0.1 * err["mixed"][0], err
