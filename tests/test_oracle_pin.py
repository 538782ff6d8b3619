"""Pin the CPU oracle against the reference's own shipped outputs.

The shipped case (flow.in: HLLC-Batten, 2nd order, CFL 0.01, 2x5 steps from a
uniform state) runs 10 steps on the merged overset mesh (266,688 tets).  The
reference wrote Velocity.dat (time and |u_g| of cell 1 per step) and
restart_files/restart0000.in (full conserved state).  The inputs (mesh and
flow.in) and the golden outputs are fixtures extracted by
tests/golden/make_golden.py, so these tests need no reference checkout.

Everything is pinned bit for bit:
  * all 10 (time, |u_g(1)|) records; cell 1 borders a corrupted overset cell
    (ghost ids of the merged mesh alias element ids, inputfiles/mergefiles.f90
    :100-110), so this pins the NaN semantics of the HLLC wave-speed MIN/MAX,
    the reuse of the previous face flux when no wave branch is taken and the
    NaN-skipping MIN of the dt reduction;
  * the set of NaN cells of the final state;
  * every finite conserved value of a 3000-cell sample and the per-variable
    sums over all finite cells;
  * a 1000-ghost sample of the ghost primitives written after the state.
Coordinates must be parsed with correct rounding (as the reference's
list-directed READ does); a 1-ulp parser breaks the match from step 2 on.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN_DIR, have_reference, shipped_case, REFERENCE_DIR


def test_fixture_equals_reference_files():
    """The committed mesh fixture decodes to exactly what the reference's
    files hold (checked where the reference checkout is mounted)."""
    if not have_reference():
        pytest.skip("HYDRA_REFERENCE_DIR not set")
    flow, mesh = shipped_case()
    flow_r, mesh_r = O.read_case_dir(REFERENCE_DIR)
    assert flow == flow_r
    for k in ("x", "y", "z", "elem", "ghost", "gid"):
        np.testing.assert_array_equal(getattr(mesh, k), getattr(mesh_r, k), err_msg=k)


@pytest.fixture(scope="module")
def shipped_run():
    flow, mesh = shipped_case()
    orc = O.Oracle(O.params_from_flow(flow), mesh)
    orc.init_uniform()
    nst = flow["niter"] * flow["itersub"]
    t, v, _ = orc.run(nst)
    cu = orc.cu()[:, :mesh.neles]
    gp = orc.ghost_restart()
    return flow, mesh, t, v, cu, gp


@pytest.mark.slow
def test_velocity_trajectory(shipped_run):
    g = np.load(os.path.join(GOLDEN_DIR, "shipped_case.npz"))
    _, _, t, v, _, _ = shipped_run
    vel = g["velocity"]
    np.testing.assert_array_equal(t, vel[:, 0])
    np.testing.assert_array_equal(v, vel[:, 1])
    assert t[-1] == float(g["restart_time"])


@pytest.mark.slow
def test_restart_state(shipped_run):
    g = np.load(os.path.join(GOLDEN_DIR, "shipped_case.npz"))
    _, mesh, _, _, cu, gp = shipped_run
    nan_cells = np.where(np.isnan(cu).any(axis=0))[0] + 1
    np.testing.assert_array_equal(nan_cells, g["nan_cells"])
    ids = g["sample_ids"] - 1
    np.testing.assert_array_equal(cu[:, ids].T, g["sample_cu"])
    sums = np.nansum(np.where(np.isnan(cu), 0.0, cu), axis=1)
    np.testing.assert_array_equal(sums, g["var_sums"])
    # ghost primitives written after the state (main.F90:819-824)
    gi = g["ghost_ids"]
    np.testing.assert_array_equal(gp[:, gi].T, g["ghost_prims"])
