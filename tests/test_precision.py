"""Precision variants against FP64 on the precision-stress case (a strong
water shock on a lattice of air bubbles), at a size the CPU oracle covers.

GPU: the FP64 parity variant equals the oracle bit for bit on it; the mixed
variant stays within 1e-5 in mixture density and pressure; the all-FP32
variant runs (it is the reference point showing what the FP64 state path
buys) and is no closer to FP64 than the mixed variant.  CPU: the EOS
recovery and positivity counts the stress report uses.
"""
import numpy as np
import pytest

import oracle as O
from hydraphase import PREC_FP32, PREC_FP64_PARITY, PREC_MIXED, Case, cases
from hydraphase.stress import errors, positivity, recover


def _spec():
    return cases.shock_lattice(nx=10, ny=10, nz=15, lattice=3, radius=0.15)


def test_recover_and_positivity():
    s = _spec()
    p, a = recover(s.cu, s.flow)
    assert np.all(p > 0) and np.all((a > 0) & (a < 1))
    assert set(np.unique(np.round(p, -3))) >= {1.0e5, 5.0e9}
    pos = positivity(s.cu, s.flow)
    assert pos == {"nan_cells": 0, "nonpositive_density": 0, "nonpositive_pressure": 0, "alpha_out_of_range": 0}
    bad = s.cu.copy()
    bad[0, 3] = -1.0
    bad[:, 7] = np.nan
    pos = positivity(bad, s.flow)
    assert pos["nan_cells"] == 1 and pos["nonpositive_density"] >= 1
    e = errors(s.cu, s.cu, s.flow)
    assert e["density"]["rel_l2"] == 0.0 and e["pressure"]["max_rel"] == 0.0


def _run(spec, prec, n):
    with Case(spec.mesh, spec.params(precision=prec)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.step(n, diagnostics=False)
        return c.state()[1]


@pytest.mark.gpu
def test_precision_variants_on_the_stress_case():
    s = _spec()
    n = 30
    m = s.mesh
    orc = O.Oracle(O.params_from_flow(s.flow, **s.extra), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
    orc.set_state(0.0, s.cu, s.ghost_prims)
    orc.run(n)
    ref = orc.cu()[:, :m.neles]
    np.testing.assert_array_equal(_run(s, PREC_FP64_PARITY, n), ref)
    mixed = _run(s, PREC_MIXED, n)
    fp32 = _run(s, PREC_FP32, n)
    em, e32 = errors(mixed, ref, s.flow), errors(fp32, ref, s.flow)
    assert em["density"]["rel_l2"] < 1e-5 and em["pressure"]["rel_l2"] < 1e-5
    assert positivity(mixed, s.flow)["nan_cells"] == 0
    assert not (e32["density"]["rel_l2"] < em["density"]["rel_l2"])
