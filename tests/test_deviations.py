"""Settings of the stated workloads that this build changes, each pinned by
the oracle (the reference's algorithm, FP64) failing at the stated setting.

Config 1 (shock-bubble, 20^3 hexes split into 6 tets):
  * as stated (air fraction 1e-6 / 1 - 1e-6, CFL 0.4) the state has NaN
    cells after the first step, in either RK scheme;
  * the contrast alone does it: at CFL 0.01 the cells on the bubble's
    interface go NaN in the first step.  A contrast of 1e-3 stays finite;
  * the CFL alone does it too: at air fraction 0.1 / 0.9, CFL 0.4 gives NaN
    cells at step 7 (the shock front).
Config 5 (precision stress, 5e9 Pa water shock on a 5 x 5 air-bubble
lattice): air bubbles at a contrast of 1e-6 (or 1e-4) give NaN cells in the
first step on a reduced 20 x 20 x 30-hex box; a contrast of 1e-3 stays
finite.
Config 2 (viscous cylinder): with the reference's convective time step
(src/main.F90:541-555) the first cell layer at the no-slip wall goes NaN at
CFL 0.5.  A reduced O-grid of the same wall spacing (40 x 64 x 4 hexes,
61,440 tets) shows it at step 157; at CFL 0.25 it stays finite.  Its
droplets as stated (alpha_w = 1 - 1e-6 inside, 1e-6 outside) give NaN cells
in the first step on the full 4,915,200-cell mesh, at CFL 0.25 too, all of
them inside droplets: the same interface contrast as config 1.
"""
import os

import numpy as np
import pytest

import oracle as O
from hydraphase import cases


def _oracle(spec, threads=1, **over):
    m = spec.mesh
    O.set_threads(threads)
    orc = O.Oracle(O.params_from_flow(spec.flow, **{**spec.extra, **over}),
                   O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    return orc


def _nan_cells(orc, neles):
    return np.isnan(orc.cu()[:, :neles]).any(axis=0)


def _centroids(m):
    el = m.elem[:, :4] - 1
    return np.stack([m.x[el].mean(1), m.y[el].mean(1), m.z[el].mean(1)], axis=1)


def _first_nan_step(orc, neles, nmax):
    for s in range(1, nmax + 1):
        orc.run(1)
        if _nan_cells(orc, neles).any():
            return s
    return None


@pytest.mark.parametrize("reference_scheme", [True, False])
def test_config1_as_stated_fails_in_first_step(reference_scheme):
    spec = cases.shock_bubble(n=20, reference_scheme=reference_scheme)
    assert spec.flow["cfl"] == 0.4 and spec.mesh.neles == 48000
    orc = _oracle(spec)
    orc.run(1)
    assert _nan_cells(orc, spec.mesh.neles).sum() > 1000
    orc.close()


def test_config1_contrast_fails_at_small_cfl_on_the_interface():
    spec = cases.shock_bubble(n=20)
    orc = _oracle(spec, cfl=0.01)
    orc.run(1)
    bad = _nan_cells(orc, spec.mesh.neles)
    orc.close()
    xc = _centroids(spec.mesh)
    r = np.linalg.norm(xc - 0.5, axis=1)
    assert bad.sum() > 1000
    assert (bad & (r > 0.15) & (r < 0.25)).sum() > 0.8 * bad.sum()    # the bubble's interface
    assert not (bad & (xc[:, 0] < 0.2)).any()                         # not the shock


def test_config1_contrast_1e3_stays_finite():
    spec = cases.shock_bubble(n=20, alpha_min=1e-3)
    orc = _oracle(spec, threads=os.cpu_count() or 1, cfl=0.05)
    assert _first_nan_step(orc, spec.mesh.neles, 10) is None
    orc.close()


def test_config1_cfl_04_fails_at_step_7():
    spec = cases.shock_bubble(n=20, alpha_min=0.1)
    orc = _oracle(spec, threads=os.cpu_count() or 1)
    assert spec.flow["cfl"] == 0.4
    assert _first_nan_step(orc, spec.mesh.neles, 10) == 7
    orc.close()


@pytest.mark.parametrize("alpha_min", [1e-6, 1e-4])
def test_config5_contrast_fails_in_first_step(alpha_min):
    spec = cases.shock_lattice(nx=20, ny=20, nz=30, alpha_min=alpha_min)
    orc = _oracle(spec, threads=os.cpu_count() or 1)
    orc.run(1)
    assert _nan_cells(orc, spec.mesh.neles).any()
    orc.close()


def test_config5_contrast_1e3_stays_finite():
    spec = cases.shock_lattice(nx=20, ny=20, nz=30, alpha_min=1e-3)
    orc = _oracle(spec, threads=os.cpu_count() or 1)
    assert _first_nan_step(orc, spec.mesh.neles, 20) is None
    orc.close()


def _reduced_cylinder():
    return cases.cylinder(nr=40, nt=64, nz=4, alpha_w_drop=1e-5)


@pytest.mark.slow
def test_cylinder_cfl05_fails_at_the_wall():
    spec = _reduced_cylinder()
    orc = _oracle(spec, threads=os.cpu_count() or 1, cfl=0.5)
    assert _first_nan_step(orc, spec.mesh.neles, 200) == 157
    bad = _nan_cells(orc, spec.mesh.neles)
    orc.close()
    xc = _centroids(spec.mesh)
    r = np.hypot(xc[:, 0], xc[:, 1])
    assert bad.any() and np.all(r[bad] < 0.505)     # first radial layer: wall at 0.5, dr0 = 0.005


@pytest.mark.slow
def test_cylinder_cfl025_stays_finite():
    spec = _reduced_cylinder()
    orc = _oracle(spec, threads=os.cpu_count() or 1, cfl=0.25)
    assert _first_nan_step(orc, spec.mesh.neles, 320) is None
    orc.close()


@pytest.mark.slow
def test_cylinder_stated_droplets_fail_in_first_step():
    spec = cases.cylinder()
    assert spec.mesh.neles == 4915200
    spec.flow["cfl"] = 0.25
    orc = _oracle(spec, threads=os.cpu_count() or 1)
    orc.run(1)
    bad = _nan_cells(orc, spec.mesh.neles)
    orc.close()
    assert bad.sum() > 10
    # the droplet centres of cases.cylinder (seed 1, 32 droplets of radius 0.1)
    rng = np.random.default_rng(1)
    dc = np.stack([rng.uniform(-8, -3, 32), rng.uniform(-2, 2, 32), rng.uniform(0.1, 3.9, 32)], axis=1)
    xc = _centroids(spec.mesh)[bad]
    dist = np.sqrt(((xc[:, None, :] - dc[None]) ** 2).sum(-1)).min(axis=1)
    assert np.all(dist < 0.1)
