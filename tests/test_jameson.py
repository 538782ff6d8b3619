"""The Jameson central flux (myflux = 3, src/sr_jameson.F90), the third
choice of the flux dispatcher (src/mod_Fluxmodule.F90:12-13): each face
takes the mean of the physical fluxes of the two cells' own states, with no
reconstruction, no limiter and no phase blending, and a wall face the phase
pressures only.  The stage calls primitiveplusbc, the central flux and the
sources; it computes no gradients.

The reference ships no run of it, so the oracle's restatement is the
reference here (parity unpinned).  CPU: properties of that restatement.
GPU: the CUDA path bit for bit against it in the FP64 parity variant, and
within the tolerances of the other flux solvers in the FMA and mixed
variants.

The central scheme carries only the JST dissipation, so the shock-bubble
box at CFL 0.4 goes non-finite after 10-13 steps in the oracle as well; the
tests run 3-5 steps of it.
"""
import numpy as np
import pytest

import oracle as O
from hydraphase import PREC_FP64, PREC_FP64_PARITY, PREC_MIXED, Case, MeshArrays, cases


def _oracle_run(spec, nsteps, **over):
    m = spec.mesh
    p = O.params_from_flow(spec.flow, **{**spec.extra, **over})
    orc = O.Oracle(p, O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    t, v, d = orc.run(nsteps)
    return t, v, d, orc.cu()[:, :m.neles], orc.ghost_restart()


def _gpu_run(spec, nsteps, precision, **over):
    with Case(spec.mesh, spec.params(precision=precision, **over)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        dg = c.step(nsteps)
        t, cu, gp = c.state()
        k = c.info()["kernels_per_step"]
    return dg, t, cu, gp, k


def _aliased(spec, shift=3, dup=(10, 11)):
    """Ghost ids shifted down so that the first ones collide with element
    ids, plus one repeated ghost id (the merged overset case's indexing)."""
    m = spec.mesh
    el, gh = m.elem.copy(), m.ghost.copy()
    new = gh[:, 1] - shift
    new[dup[0]] = new[dup[1]]
    for g in range(gh.shape[0]):
        p, side = gh[g, 0] - 1, gh[g, 3] - 1
        el[p, 4 + side] = new[g]
    gh[:, 1] = new
    spec.mesh = MeshArrays(m.x, m.y, m.z, el, gh)
    return spec


SPECS = {
    "shock_bubble_ref": lambda: cases.shock_bubble(n=5, alpha_min=0.1, reference_scheme=True),
    "shock_bubble_ext": lambda: cases.shock_bubble(n=5, alpha_min=0.1, reference_scheme=False),
    "cylinder": lambda: cases.cylinder(nr=6, nt=16, nz=2),
    "aliased_ghosts": lambda: _aliased(cases.shock_bubble(n=5, alpha_min=0.1, reference_scheme=True)),
}


# ---------------------------------------------------------------- CPU


def test_oracle_rest_box_stays_at_rest():
    """Gas and liquid at rest at uniform pressure in a closed box (walls of
    type 5): the central fluxes of equal states reduce to the pressure
    terms, which cancel over each closed cell to rounding.  The momenta
    stay at the level HLLC-Batten leaves them at (rounding of the pressure
    terms on the jittered cells) and the masses within 1e-6."""
    b = cases.box_mesh(4, 4, 4, jitter=0.1, seed=3, bc_type=5)
    sp = cases.shock_bubble_on(b, p_post=1e5, rho_post=1000.0, post_velocity=0.0, alpha_min=0.5)
    _, _, _, cu, _ = _oracle_run(sp, 10, myflux=3)
    _, _, _, cu_b, _ = _oracle_run(sp, 10, myflux=2)
    assert np.isfinite(cu).all()
    mom = [1, 2, 3, 6, 7, 8]
    assert np.abs(cu[mom]).max() < 2 * np.abs(cu_b[mom]).max()
    np.testing.assert_allclose(cu[[0, 5]], sp.cu[[0, 5]], rtol=1e-6)


def test_oracle_jameson_is_its_own_solver():
    spec = SPECS["cylinder"]()
    _, _, _, cu3, _ = _oracle_run(spec, 10, myflux=3)
    _, _, _, cu2, _ = _oracle_run(spec, 10, myflux=2)
    assert np.isfinite(cu3).all()
    assert not np.array_equal(cu3, cu2)


def test_oracle_rejects_unknown_flux():
    spec = SPECS["cylinder"]()
    m = spec.mesh
    with pytest.raises(ValueError, match="myflux"):
        O.Oracle(O.params_from_flow(spec.flow, **{**spec.extra, "myflux": 4}),
                 O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))


# ---------------------------------------------------------------- GPU


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SPECS))
def test_jameson_fp64_parity_bit_exact(name):
    spec = SPECS[name]()
    n = 3
    t, v, d, cu_o, gp_o = _oracle_run(spec, n, myflux=3)
    dg, tg, cu_g, gp_g, k = _gpu_run(spec, n, PREC_FP64_PARITY, myflux=3)
    np.testing.assert_array_equal(dg["time"], t)
    np.testing.assert_array_equal(dg["velmag"], v)
    np.testing.assert_array_equal(dg["diff"], d)
    np.testing.assert_array_equal(cu_g, cu_o)
    np.testing.assert_array_equal(gp_g, gp_o)
    if name != "aliased_ghosts":
        # no gradient kernel in the stage
        _, _, _, _, k2 = _gpu_run(spec, 1, PREC_FP64_PARITY, myflux=2)
        stages = 4 if spec.extra.get("rk_scheme", 0) == 0 else 3
        assert k == k2 - stages


@pytest.mark.gpu
def test_jameson_fp64_parity_renumbered_and_graph_modes():
    """Cells renumbered along the Hilbert curve, and the separate launches,
    the graph and a fused-step request (which keeps the graph for this
    flux), all bit-identical to the oracle."""
    spec = SPECS["cylinder"]()
    _, _, _, cu_o, _ = _oracle_run(spec, 4, myflux=3)
    for over in ({"renumber": 1}, {"use_graph": 0}, {"use_graph": 1}, {"use_graph": 2}):
        _, _, cu_g, _, _ = _gpu_run(spec, 4, PREC_FP64_PARITY, myflux=3, **over)
        np.testing.assert_array_equal(cu_g, cu_o, err_msg=str(over))


@pytest.mark.gpu
def test_jameson_fp64_fma_within_1e10():
    """As for HLLC: the air variables within 1e-10; the trace water phase
    (alpha_w = 1e-6, recovered as 1 - alpha_g) within 1e-4."""
    spec = SPECS["cylinder"]()
    _, _, _, cu_o, _ = _oracle_run(spec, 5, myflux=3)
    _, _, cu_g, _, _ = _gpu_run(spec, 5, PREC_FP64, myflux=3)
    err = np.linalg.norm(cu_g - cu_o, axis=1) / np.linalg.norm(cu_o, axis=1)
    assert np.all(err[:5] < 1e-10), err
    assert np.all(err[5:] < 1e-4), err


@pytest.mark.gpu
@pytest.mark.parametrize("face_mode", [0, 1, 2, 3])
def test_jameson_mixed_within_tolerance(face_mode):
    spec = SPECS["cylinder"]()
    _, _, _, cu_o, _ = _oracle_run(spec, 5, myflux=3)
    _, _, cu_g, _, _ = _gpu_run(spec, 5, PREC_MIXED, myflux=3, face_mode=face_mode)
    rho_o, rho_g = cu_o[0] + cu_o[5], cu_g[0] + cu_g[5]
    assert np.linalg.norm(rho_g - rho_o) / np.linalg.norm(rho_o) < 1e-5


@pytest.mark.gpu
def test_jameson_wall_layers_cover_every_cell():
    """Mixed with every cell in the FP64 wall layers is the FP64 variant bit
    for bit with this flux too."""
    spec = SPECS["cylinder"]()
    _, _, cu64, _, _ = _gpu_run(spec, 5, PREC_FP64, myflux=3)
    _, _, cuw, _, _ = _gpu_run(spec, 5, PREC_MIXED, myflux=3, wall_fp64_layers=1 << 20)
    np.testing.assert_array_equal(cuw, cu64)


@pytest.mark.gpu
def test_jameson_five_phase_matches_oracle():
    """The five-phase equations (the dispersed phases' own central fluxes
    come after CallFluxSolver, src/mod_Fluxmodule.F90:18-20) with the
    Jameson flux for the two-phase rows: the five-phase bar of 1e-12
    relative L2 per variable (the drag law's pow differs between libm and
    CUDA in the last bit)."""
    base = cases.shock_bubble(n=5, alpha_min=0.1, reference_scheme=True)
    base.flow["cfl"] = 0.1
    spec = cases.with_dispersed(base, rad=(2.0e-4, 4.0e-4, 3.0e-4))
    _, _, _, cu_o, _ = _oracle_run(spec, 5, myflux=3)
    _, _, cu_g, _, _ = _gpu_run(spec, 5, PREC_FP64_PARITY, myflux=3)
    assert cu_g.shape == (22, spec.mesh.neles) and np.isfinite(cu_g).all()
    err = np.linalg.norm(cu_g - cu_o, axis=1) / np.linalg.norm(cu_o, axis=1)
    assert np.all(err < 1e-12), err
