"""The five-phase model (the reference's FIVE_PHASE build): three dispersed,
incompressible particle phases q, r, s with mass and momentum each (22
conserved variables), central fluxes (src/sr_jamesonqrs.F90), their JST
dissipation (src/sr_dissipationqrs.F90) and drag on the liquid
(src/sr_sourceqrs.F90), and the dispersed volume taken out of the
pressure-equilibrium recovery (src/sr_primitive.F90:56-80).

The reference ships no five-phase run, so the oracle's restatement is the
reference here (parity unpinned).  CPU: properties of that restatement and the
engine's argument checks.  GPU: the CUDA path against the oracle.  The drag
coefficient uses pow(Re, 0.85) (libm in the oracle, CUDA's pow on the
device), which may differ in the last bit, so the GPU bar is 1e-12 relative
L2 per variable instead of bit equality.

The cases are shock-bubble boxes with particles of 0.2-0.4 mm: with the
shipped radii (5-20 um) and the liquid viscosity 0.001 of the reference, the
particles relax to the liquid velocity within ~1e-5 s, and the explicit
scheme is stable only at time steps below that.
"""
import numpy as np
import pytest

import oracle as O
from hydraphase import PREC_FP32, PREC_FP64_PARITY, PREC_MIXED, Case, HP_E_ARG, HP_E_UNSUPPORTED, HydraError, cases

RAD = (2.0e-4, 4.0e-4, 3.0e-4)


def _spec(reference_scheme=True, n=5):
    base = cases.shock_bubble(n=n, alpha_min=0.1, reference_scheme=reference_scheme)
    base.flow["cfl"] = 0.1
    return cases.with_dispersed(base, rad=RAD)


def _oracle(spec, **over):
    m = spec.mesh
    orc = O.Oracle(O.params_from_flow(spec.flow, **{**spec.extra, **over}), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    return orc


def _rest_box():
    """Liquid and gas at rest at uniform pressure in a closed box, uniform
    dispersed fractions: an equilibrium of the model."""
    b = cases.box_mesh(4, 4, 4, jitter=0.1, seed=3, bc_type=5)
    sp0 = cases.shock_bubble_on(b, p_post=1e5, rho_post=1000.0, post_velocity=0.0, alpha_min=0.5)
    sp = cases.with_dispersed(sp0, slip=0.0, rad=RAD)
    frac, rho = (2e-3, 1e-3, 5e-4), (2500.0, 1950.0, 2700.0)
    sp.cu[:10] = sp0.cu * (1.0 - sum(frac))
    for d in range(3):
        sp.cu[10 + 4 * d] = frac[d] * rho[d]
        sp.cu[11 + 4 * d:14 + 4 * d] = 0.0
    return sp0, sp


def test_oracle_rest_state_stays_at_rest():
    sp0, sp = _rest_box()
    out = []
    for s in (sp0, sp):
        orc = _oracle(s)
        orc.run(10)
        out.append(orc.cu()[:, :s.mesh.neles])
    two, five = out
    assert five.shape[0] == 22
    # the two-phase variables move exactly as much as in the two-phase model
    # at rest (rounding only), and the dispersed masses stay put
    mom = [1, 2, 3, 6, 7, 8]
    assert np.abs(five[mom]).max() < 10 * max(np.abs(two[mom]).max(), 1e-12)
    for d in range(3):
        np.testing.assert_allclose(five[10 + 4 * d], sp.cu[10 + 4 * d], rtol=1e-10)
        assert np.abs(five[11 + 4 * d:14 + 4 * d]).max() < 1e-6


def test_oracle_dispersed_phases_move_and_stay_finite():
    spec = _spec()
    orc = _oracle(spec)
    orc.run(10)
    cu = orc.cu()[:, :spec.mesh.neles]
    assert np.isfinite(cu).all()
    # the shock drags the liquid, the liquid drags the particles
    assert np.abs(cu[11] - spec.cu[11]).max() > 1e-3 * np.abs(spec.cu[11]).max()


def test_create_checks_five_phase_arguments():
    spec = _spec(n=2)
    with pytest.raises(HydraError) as e:
        Case(spec.mesh, spec.params(rhoq=0.0))
    assert e.value.code == HP_E_ARG
    with pytest.raises(HydraError) as e:
        Case(spec.mesh, spec.params(precision=PREC_FP32))
    assert e.value.code == HP_E_UNSUPPORTED


def _rel_l2(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("reference_scheme", [True, False])
def test_five_phase_gpu_matches_oracle(reference_scheme):
    spec = _spec(reference_scheme)
    orc = _oracle(spec)
    t, v, _ = orc.run(10)
    cu_o = orc.cu()[:, :spec.mesh.neles]
    gp_o = orc.ghost_restart()
    with Case(spec.mesh, spec.params(precision=PREC_FP64_PARITY)) as c:
        assert c.info()["kernels_per_step"] > 0
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        dg = c.step(10)
        _, cu_g, gp_g = c.state()
    assert cu_g.shape == (22, spec.mesh.neles)
    assert np.isfinite(cu_g).all()
    err = _rel_l2(cu_g, cu_o)
    assert np.all(err < 1e-12), err
    np.testing.assert_allclose(dg["time"], t, rtol=1e-13)
    assert np.all(_rel_l2(gp_g, gp_o) < 1e-12)


@pytest.mark.gpu
def test_five_phase_mixed_within_tolerance():
    spec = _spec(True)
    orc = _oracle(spec)
    orc.run(5)
    cu_o = orc.cu()[:, :spec.mesh.neles]
    with Case(spec.mesh, spec.params(precision=PREC_MIXED)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.step(5)
        _, cu_g, _ = c.state()
    rho_o, rho_g = cu_o[0] + cu_o[5], cu_g[0] + cu_g[5]
    assert np.linalg.norm(rho_g - rho_o) / np.linalg.norm(rho_o) < 1e-4
    for d in range(3):
        k = 10 + 4 * d
        assert np.linalg.norm(cu_g[k] - cu_o[k]) / np.linalg.norm(cu_o[k]) < 1e-4
