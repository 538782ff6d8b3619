"""Overset fringe interpolation (new work; the reference only freezes cells
with iblank != 1 and takes its donors from TIOGA).

CPU: the library's fringe and donor tables (hp_overset_build) equal the
oracle's restatement bit for bit; fringe cells are the field cells next to
holes / the component's outer boundary; donors are field cells of the other
block; weights sum to one and reproduce linear fields.
GPU: steps with the table attached (fringe cells interpolated after every RK
stage) equal the oracle bit for bit in the FP64 parity variant, and the mixed
variant stays within 1e-5 in mixture density and alpha_g; the device builder
(hp_overset_build_gpu) returns the host builder's tables bit for bit,
nearest-centroid fallbacks included.
Hole cut: background cells within a margin of, or enclosed by, the
component's wall faces; the library equals the oracle and the geometric
answer on CPU (rays through shared edges and vertices counted once), and the
device cut equals the host's.
"""
import numpy as np
import pytest

import oracle as O
from hydraphase import HP_E_UNSUPPORTED, PREC_FP64_PARITY, PREC_MIXED, Batch, Case, HydraError, cases
from hydraphase.engine import MeshArrays, overset_build, overset_hole_cut


def _small():
    return cases.overset_cylinder(bg=(24, 24, 2), comp=(12, 48, 2), box=((-6.0, -6.0, 0.0), (6.0, 6.0, 4.0)),
                                  alpha_w_drop=1e-5, alpha_w_bg=1e-6)


def _with_iblank(mesh, ib):
    el = mesh.elem.copy()
    el[:, 8] = ib
    return MeshArrays(mesh.x, mesh.y, mesh.z, el, mesh.ghost)


def test_tables_equal_oracle_and_are_consistent():
    ov = _small()
    m = ov.spec.mesh
    ib, tab = overset_build(m, ov.block, ov.layers, ov.outer_type)
    ib2, fr2, dn2, w2, nfb2 = O.overset_build(O.Mesh(m.x, m.y, m.z, m.elem, m.ghost), ov.block, ov.layers,
                                              ov.outer_type)
    np.testing.assert_array_equal(ib, ib2)
    np.testing.assert_array_equal(tab.fringe, fr2)
    np.testing.assert_array_equal(tab.donor, dn2)
    np.testing.assert_array_equal(tab.weight, w2)
    assert tab.nfallback == nfb2 == 0
    assert tab.fringe.size > 0 and np.all(ib[tab.fringe - 1] == -1) and (ib == -1).sum() == tab.fringe.size
    assert np.all(ib[m.elem[:, 8] == 0] == 0)                       # holes stay holes
    blk = ov.block
    for f, d in zip(tab.fringe, tab.donor):
        assert np.all(ib[d - 1] == 1) and np.all(blk[d - 1] == 1 - blk[f - 1])
    np.testing.assert_allclose(tab.weight.sum(axis=1), 1.0, rtol=0, atol=1e-13)
    x = m.x[m.elem[:, :4] - 1]
    xc = 0.25 * (x[:, 0] + x[:, 1] + x[:, 2] + x[:, 3])
    f = 0.3 * xc + 2.0
    np.testing.assert_allclose((tab.weight * f[tab.donor - 1]).sum(axis=1), f[tab.fringe - 1], rtol=0, atol=1e-12)
    assert tab.weight.min() > -0.5                                  # mild extrapolation at most


def test_fringe_layers_grow_inward():
    ov = _small()
    m = ov.spec.mesh
    _, t1 = overset_build(m, ov.block, 1, ov.outer_type)
    _, t2 = overset_build(m, ov.block, 2, ov.outer_type)
    assert set(t1.fringe) < set(t2.fringe)


def _oracle(spec, mesh, tab, n):
    orc = O.Oracle(O.params_from_flow(spec.flow, **spec.extra), O.Mesh(mesh.x, mesh.y, mesh.z, mesh.elem, mesh.ghost))
    orc.set_state(0.0, spec.cu, spec.ghost_prims)
    orc.set_overset(tab.fringe, tab.donor, tab.weight)
    t, v, d = orc.run(n)
    return t, orc.cu()[:, :mesh.neles], orc.ghost_restart()


@pytest.mark.gpu
@pytest.mark.parametrize("renumber", [0, 1])
def test_overset_steps_bit_exact(renumber):
    ov = _small()
    spec = ov.spec
    ib, tab = overset_build(spec.mesh, ov.block, ov.layers, ov.outer_type)
    mesh = _with_iblank(spec.mesh, ib)
    n = 4
    t, cu_o, gp_o = _oracle(spec, mesh, tab, n)
    with Case(mesh, spec.params(precision=PREC_FP64_PARITY, renumber=renumber)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.set_overset(tab)
        d = c.step(n)
        _, cu, gp = c.state()
    np.testing.assert_array_equal(d["time"], t)
    np.testing.assert_array_equal(cu, cu_o)
    np.testing.assert_array_equal(gp, gp_o)


@pytest.mark.gpu
def test_overset_mixed_within_tolerance():
    ov = _small()
    spec = ov.spec
    ib, tab = overset_build(spec.mesh, ov.block, ov.layers, ov.outer_type)
    mesh = _with_iblank(spec.mesh, ib)
    _, cu_o, _ = _oracle(spec, mesh, tab, 5)
    with Case(mesh, spec.params(precision=PREC_MIXED)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.set_overset(tab)
        c.step(5, diagnostics=False)
        _, cu, _ = c.state()
    rho_o, rho = cu_o[0] + cu_o[5], cu[0] + cu[5]
    assert np.linalg.norm(rho - rho_o) / np.linalg.norm(rho_o) < 1e-5


@pytest.mark.gpu
def test_overset_table_rejected_on_batches():
    ov = _small()
    spec = ov.spec
    ib, tab = overset_build(spec.mesh, ov.block, ov.layers, ov.outer_type)
    mesh = _with_iblank(spec.mesh, ib)
    with Batch([mesh, mesh], spec.params()) as b:
        from hydraphase.engine import _check  # noqa: F401
        import ctypes
        from hydraphase._lib import HpOverset, lib
        fr = np.ascontiguousarray(tab.fringe, np.int32)
        dn = np.ascontiguousarray(tab.donor, np.int32).ravel()
        w = np.ascontiguousarray(tab.weight).ravel()
        o = HpOverset(fr.size, fr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      dn.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0)
        assert lib().hp_set_overset(b.h, ctypes.byref(o)) == HP_E_UNSUPPORTED


@pytest.mark.gpu
@pytest.mark.parametrize("layers", [1, 2])
def test_device_tables_equal_host(layers):
    """hp_overset_build_gpu returns the host builder's tables bit for bit."""
    ov = _small()
    m = ov.spec.mesh
    ib_h, th = overset_build(m, ov.block, layers, ov.outer_type)
    ib_d, td = overset_build(m, ov.block, layers, ov.outer_type, device=True)
    np.testing.assert_array_equal(ib_h, ib_d)
    np.testing.assert_array_equal(th.fringe, td.fringe)
    np.testing.assert_array_equal(th.donor, td.donor)
    np.testing.assert_array_equal(th.weight, td.weight)
    assert th.nfallback == td.nfallback


@pytest.mark.gpu
def test_device_tables_with_nearest_fallback():
    """A component that reaches beyond the background: its outer fringe lies
    in no background tet, so the nearest-centroid fallback runs; host and
    device agree on it too."""
    ov = cases.overset_cylinder(bg=(12, 12, 2), comp=(8, 32, 2), box=((-2.5, -2.5, 0.0), (2.5, 2.5, 4.0)),
                                alpha_w_drop=1e-5, alpha_w_bg=1e-6)
    m = ov.spec.mesh
    ib_h, th = overset_build(m, ov.block, ov.layers, ov.outer_type)
    ib_d, td = overset_build(m, ov.block, ov.layers, ov.outer_type, device=True)
    assert th.nfallback > 0
    np.testing.assert_array_equal(ib_h, ib_d)
    np.testing.assert_array_equal(th.fringe, td.fringe)
    np.testing.assert_array_equal(th.donor, td.donor)
    np.testing.assert_array_equal(th.weight, td.weight)
    assert th.nfallback == td.nfallback


# --- hole cut (hp_overset_hole_cut / _gpu) ------------------------------------
def _cube_in_box():
    """A unit cube of wall faces (component, 2x2x2 hexes, type 6) inside a
    background box whose tet centroids put many +x rays exactly through the
    cube's face edges and vertices (y, z on multiples of 1/8; cube nodes at
    multiples of 1/2); no centroid lies on the cube's surface."""
    bg = cases.box_mesh(10, 10, 10, lo=(-2.05, -2.0, -2.0), hi=(2.95, 3.0, 3.0), bc_type=7)
    cube = cases.box_mesh(2, 2, 2, bc_type=6)
    u, block = cases.union_mesh(bg, cube)
    return u, block


def _unblanked(mesh):
    el = mesh.elem.copy()
    el[:, 8] = 1
    return MeshArrays(mesh.x, mesh.y, mesh.z, el, mesh.ghost)


@pytest.mark.parametrize("margin", [0.0, 0.3])
def test_hole_cut_cube_equals_geometry_and_oracle(margin):
    """Holes are exactly the background cells inside the cube or within the
    margin of it (Euclidean distance to the solid cube), rays through shared
    edges and vertices included; the library equals the oracle."""
    u, block = _cube_in_box()
    ib, nh = overset_hole_cut(u.mesh, block, wall_type=6, margin=margin)
    ib_o, nh_o = O.overset_hole_cut(O.Mesh(u.mesh.x, u.mesh.y, u.mesh.z, u.mesh.elem, u.mesh.ghost), block, 6,
                                    margin)
    xc = u.xc
    gap = np.maximum(0.0, np.maximum(-xc, xc - 1.0))
    inside = np.all((xc > 0.0) & (xc < 1.0), axis=1)
    expect = (block == 0) & (inside | (np.sqrt((gap ** 2).sum(axis=1)) <= margin))
    np.testing.assert_array_equal(ib == 0, expect)
    np.testing.assert_array_equal(ib, ib_o)
    assert nh == nh_o == expect.sum() > 0


@pytest.mark.parametrize("sizes", [((24, 24, 2), (12, 48, 2)), ((40, 30, 3), (16, 64, 3))])
def test_hole_cut_cylinder_equals_radius_rule(sizes):
    """Within hole_r - 0.5 of the cylinder's wall faces or inside them: the
    same holes as the radius rule r < hole_r on these meshes (no centroid in
    the band where the polygonal wall departs from the circle), equal to the
    oracle, background field cells only."""
    bg, comp = sizes
    box = ((-6.0, -6.0, 0.0), (6.0, 6.0, 4.0))
    ovr = cases.overset_cylinder(bg=bg, comp=comp, box=box)
    ovw = cases.overset_cylinder(bg=bg, comp=comp, box=box, hole_cut="wall")
    np.testing.assert_array_equal(ovr.spec.mesh.elem[:, 8], ovw.spec.mesh.elem[:, 8])
    m = _unblanked(ovr.spec.mesh)
    ib, nh = overset_hole_cut(m, ovr.block, wall_type=6, margin=0.7)
    ib_o, nh_o = O.overset_hole_cut(O.Mesh(m.x, m.y, m.z, m.elem, m.ghost), ovr.block, 6, 0.7)
    np.testing.assert_array_equal(ib, ib_o)
    assert nh == nh_o == (ib == 0).sum() > 0 and np.all(ovr.block[ib == 0] == 0)
    ib0, _ = overset_hole_cut(m, ovr.block, wall_type=6, margin=0.0)     # the body alone
    xc = ovr.spec.mesh.x[m.elem[:, :4] - 1].mean(axis=1), ovr.spec.mesh.y[m.elem[:, :4] - 1].mean(axis=1)
    r = np.hypot(*xc)
    assert np.all(r[ib0 == 0] < 0.5) and np.all(ib0[(ovr.block == 0) & (r < 0.49)] == 0)


def test_hole_cut_rejects_bad_arguments():
    u, block = _cube_in_box()
    with pytest.raises(HydraError):
        overset_hole_cut(u.mesh, block, wall_type=6, margin=-1.0)
    with pytest.raises(HydraError):
        overset_hole_cut(u.mesh, block, wall_type=99, margin=0.0)       # no wall face of that type
    bad = block.copy()
    bad[0] = 2
    with pytest.raises(HydraError):
        overset_hole_cut(u.mesh, bad, wall_type=6, margin=0.0)


@pytest.mark.gpu
def test_hole_cut_device_equals_host():
    """hp_overset_hole_cut_gpu returns the host's iblank bit for bit, and the
    whole device chain (hole cut, donor search) gives the host chain's
    tables."""
    u, block = _cube_in_box()
    for margin in (0.0, 0.3):
        ib_h, nh_h = overset_hole_cut(u.mesh, block, 6, margin)
        ib_d, nh_d = overset_hole_cut(u.mesh, block, 6, margin, device=True)
        np.testing.assert_array_equal(ib_h, ib_d)
        assert nh_h == nh_d
    ov = cases.overset_cylinder(bg=(40, 30, 3), comp=(16, 64, 3), box=((-6.0, -6.0, 0.0), (6.0, 6.0, 4.0)))
    m = _unblanked(ov.spec.mesh)
    ib_h, nh_h = overset_hole_cut(m, ov.block, 6, 0.7)
    ib_d, nh_d = overset_hole_cut(m, ov.block, 6, 0.7, device=True)
    np.testing.assert_array_equal(ib_h, ib_d)
    assert nh_h == nh_d > 0
    mh = _with_iblank(m, ib_h)
    fh, th = overset_build(mh, ov.block, ov.layers, ov.outer_type)
    fd, td = overset_build(_with_iblank(m, ib_d), ov.block, ov.layers, ov.outer_type, device=True)
    np.testing.assert_array_equal(fh, fd)
    np.testing.assert_array_equal(th.donor, td.donor)
    np.testing.assert_array_equal(th.weight, td.weight)
