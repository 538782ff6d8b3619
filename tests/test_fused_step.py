"""The fused step (hp_params.use_graph = 2): one cooperative kernel runs a
whole time step, the step's kernels as phases over virtual blocks with
grid-wide barriers between them.  In the parity variant it must give the
separate launches' results bit for bit, in both RK schemes and both HLLC
solvers.  The variants built with FMA contraction keep the graph (another
compilation of the same bodies may contract, and so round, differently):
there use_graph = 2 runs exactly as 1."""
import numpy as np
import pytest

from hydraphase import (HP_E_ARG, PREC_FP64, PREC_FP64_PARITY, PREC_MIXED, Case, HydraError, cases)


def _steps(spec, n, **over):
    with Case(spec.mesh, spec.params(**over)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        d = c.step(n)
        _, cu, gp = c.state()
        k = c.info()["kernels_per_step"]
    return cu, gp, d, k


def test_use_graph_values_checked():
    spec = cases.shock_bubble(n=2)
    with pytest.raises(HydraError) as e:
        Case(spec.mesh, spec.params(use_graph=3))
    assert e.value.code == HP_E_ARG and "use_graph" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("reference_scheme", [True, False])
def test_fused_step_equals_separate_launches(reference_scheme):
    spec = cases.shock_bubble(n=8, alpha_min=0.1, reference_scheme=reference_scheme)
    spec.flow["cfl"] = 0.05
    a = _steps(spec, 12, precision=PREC_FP64_PARITY, use_graph=1)
    b = _steps(spec, 12, precision=PREC_FP64_PARITY, use_graph=2)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[1], a[1])
    for key in ("time", "dt", "velmag", "diff", "nan_cells"):
        np.testing.assert_array_equal(b[2][key], a[2][key])
    assert b[3] == 1 and a[3] > 10


@pytest.mark.gpu
@pytest.mark.parametrize("myflux", [1, 2])
def test_fused_step_viscous_cylinder(myflux):
    spec = cases.cylinder(nr=12, nt=32, nz=4, alpha_w_drop=1e-5, alpha_w_bg=1e-6)
    spec.flow["cfl"] = 0.25
    a = _steps(spec, 20, precision=PREC_FP64_PARITY, myflux=myflux, use_graph=1)
    b = _steps(spec, 20, precision=PREC_FP64_PARITY, myflux=myflux, use_graph=2)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[2]["dt"], a[2]["dt"])
    assert b[3] == 1


@pytest.mark.gpu
def test_fused_step_batch_equals_separate_launches():
    specs = [cases.shock_bubble(n=n, alpha_min=0.1, seed=n) for n in (4, 6, 5)]
    from hydraphase import Batch
    out = []
    for g in (1, 2):
        with Batch([sp.mesh for sp in specs], specs[0].params(precision=PREC_FP64_PARITY, cfl=0.05, use_graph=g)) as b:
            for k, sp in enumerate(specs):
                b.set_state(k, 0.0, sp.cu, sp.ghost_prims)
            b.step(8, diagnostics=False)
            out.append([b.state(k)[1] for k in range(len(specs))])
    for x, y in zip(out[1], out[0]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,over", [(PREC_FP64, {}), (PREC_MIXED, {}),
                                       (PREC_MIXED, {"wall_fp64_layers": 4})])
def test_other_handles_keep_the_graph(prec, over):
    spec = cases.cylinder(nr=12, nt=32, nz=4, alpha_w_drop=1e-5, alpha_w_bg=1e-6)
    spec.flow["cfl"] = 0.25
    a = _steps(spec, 5, precision=prec, use_graph=1, **over)
    b = _steps(spec, 5, precision=prec, use_graph=2, **over)
    np.testing.assert_array_equal(b[0], a[0])
    assert b[3] == a[3] > 1
