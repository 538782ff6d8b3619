"""Multi-mesh batches (hp_create_batch): the cell and ghost lists of several
cases concatenated in one handle, one kernel sweep per step for all of them.

GPU: each case of a batch ends bit-identical to the same case alone and, for
the FP64 parity variant, to the oracle; per-case diagnostics match; a batch's
states cannot be replaced after its first step.  CPU: argument checks that
happen before any device work, and the byte estimate.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from hydraphase import (HP_E_CUDA, HP_E_STATE, HP_E_UNSUPPORTED, PREC_FP64_PARITY, PREC_MIXED, Batch, Case,
                        HydraError, MeshArrays, cases)
from hydraphase.engine import estimate_batch_bytes, estimate_bytes


def _members():
    """Shock-bubble cases of different sizes, meshes and states that share
    one set of flow parameters (a batch has one)."""
    out = []
    for n, r, pp, seed in ((4, 0.2, 1e9, 0), (5, 0.25, 3e8, 1), (3, 0.15, 2e9, 2), (6, 0.3, 1e8, 3)):
        b = cases.box_mesh(n, n, n, jitter=0.1, seed=seed, bc_type=5)
        out.append(cases.shock_bubble_on(b, radius=r, p_post=pp, alpha_min=0.1))
    return out


def _aliased_mesh(spec):
    m = spec.mesh
    el, gh = m.elem.copy(), m.ghost.copy()
    new = gh[:, 1] - 3
    for g in range(gh.shape[0]):
        el[gh[g, 0] - 1, 4 + gh[g, 3] - 1] = new[g]
    gh[:, 1] = new
    return MeshArrays(m.x, m.y, m.z, el, gh)


def test_batch_rejects_aliased_member():
    s = _members()
    with pytest.raises(HydraError) as e:
        Batch([s[0].mesh, _aliased_mesh(s[1])], s[0].params())
    assert e.value.code == HP_E_UNSUPPORTED and "batch" in str(e.value)


def test_batch_estimate_close_to_sum_of_members():
    s = _members()
    p = s[0].params(precision=PREC_MIXED)
    tot = estimate_batch_bytes([x.mesh for x in s], p)
    parts = sum(estimate_bytes(x.mesh, p) for x in s)
    assert 0.9 * parts < tot <= parts


def test_batch_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    s = _members()
    with pytest.raises(HydraError) as e:
        Batch([x.mesh for x in s], s[0].params())
    assert e.value.code == HP_E_CUDA


def _alone(spec, params, n):
    with Case(spec.mesh, params) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        d = c.step(n)
        return d, c.state()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_FP64_PARITY, PREC_MIXED])
def test_batch_members_equal_alone(precision):
    s = _members()
    p = s[0].params(precision=precision)
    n = 4
    with Batch([x.mesh for x in s], p) as b:
        for k, x in enumerate(s):
            b.set_state(k, 0.0, x.cu, x.ghost_prims)
        diags = b.step(n)
        got = [b.state(k) for k in range(len(s))]
        with pytest.raises(HydraError) as e:
            b.set_state(0, 0.0, s[0].cu, s[0].ghost_prims)
        assert e.value.code == HP_E_STATE
    for k, x in enumerate(s):
        d, (t, cu, gp) = _alone(x, p, n)
        np.testing.assert_array_equal(diags[k]["time"], d["time"])
        np.testing.assert_array_equal(diags[k]["velmag"], d["velmag"])
        np.testing.assert_array_equal(diags[k]["diff"], d["diff"])
        assert got[k][0] == t
        np.testing.assert_array_equal(got[k][1], cu)
        np.testing.assert_array_equal(got[k][2], gp)


@pytest.mark.gpu
def test_batch_parity_against_oracle():
    s = _members()
    p = s[0].params(precision=PREC_FP64_PARITY)
    n = 3
    with Batch([x.mesh for x in s], p) as b:
        for k, x in enumerate(s):
            b.set_state(k, 0.0, x.cu, x.ghost_prims)
        b.step(n, diagnostics=False)
        got = [b.state(k) for k in range(len(s))]
    for k, x in enumerate(s):
        m = x.mesh
        orc = O.Oracle(O.params_from_flow(x.flow, **x.extra), O.Mesh(m.x, m.y, m.z, m.elem, m.ghost))
        orc.set_state(0.0, x.cu, x.ghost_prims)
        orc.run(n)
        np.testing.assert_array_equal(got[k][1], orc.cu()[:, :m.neles])
        np.testing.assert_array_equal(got[k][2], orc.ghost_restart())
