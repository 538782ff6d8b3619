"""Output in the reference's formats: the Tecplot file of src/main.F90:956-1268
and asynchronous output (hp_output_async) that overlaps later steps.

CPU: hp_write_tecplot writes the reference's header, zone line, node
coordinates, 13 cell-centred fields and connectivity, every value as Fortran
ES16.8 (checked against a Python restatement of the edit descriptor).
GPU: a snapshot taken between steps and written while later steps run is the
same restart file as hp_get_state + hp_write_restart at that point, and its
Tecplot fields equal a plain FP64 evaluation of src/main.F90:996-1131 on the
snapshot's state, character for character.
"""
import ctypes
import math

import numpy as np
import pytest

from hydraphase import PREC_FP64_PARITY, PREC_MIXED, Case, cases, lib
from hydraphase.engine import write_tecplot

HEADER = (' VARIABLES = "X", "Y", "Z", "U","V", "W", "PG", "PP", "TG", "UP", "VP", "WP", "PHIG", "TP", "ROG", '
          '"ROP"')


def es16_8(v: float) -> str:
    """Fortran ES16.8: d.dddddddd, exponent with E for two digits, without
    it for three, right-justified in 16 columns."""
    if math.isnan(v):
        s = "NaN"
    elif math.isinf(v):
        s = "Infinity" if v > 0 else "-Infinity"
    else:
        s = "%.8E" % v
        mant, exp = s.split("E")
        if len(exp) == 4:
            s = mant + exp
    return s.rjust(16)


def expected_tecplot(mesh, fields) -> str:
    ne, nn = mesh.neles, mesh.nodes
    lines = [HEADER, f"ZONE ZONETYPE=FETETRAHEDRON, NODES={nn}, ELEMENTS={ne}, DATAPACKING=BLOCK, "
                     f"VARLOCATION=([4-16]=CELLCENTERED)"]
    for col in (mesh.x, mesh.y, mesh.z):
        lines += [es16_8(float(v)) for v in col]
    for k in range(13):
        lines += [es16_8(float(v)) for v in fields[k]]
    lines += ["%12d%12d%12d%12d" % tuple(r[:4]) for r in mesh.elem]
    return "\n".join(lines) + "\n"


def tecplot_fields(cu, flow):
    """src/main.F90:996-1131, two-phase branch, in its operation order."""
    gg, gp, pinf = flow["gamag"], flow["gamap"], flow["pinf"]
    fs = 4.0 * flow["surfacetension"] / flow["diap"]
    emin, emax, rrg, cpp = flow["epslnmin"], flow["epslnmax"], 287.0, flow["cpp"]
    c = [cu[k].astype(np.float64) for k in range(10)]
    ug, vg, wg = c[1] / c[0], c[2] / c[0], c[3] / c[0]
    up, vp, wp = c[6] / c[5], c[7] / c[5], c[8] / c[5]
    eg = c[4] / c[0] - 0.5 * (ug * ug + vg * vg + wg * wg)
    ep = c[9] / c[5] - 0.5 * (up * up + vp * vp + wp * wp)
    bbb = (fs + pinf * gp) - (c[0] * (gg - 1.0) * eg) - (c[5] * (gp - 1.0) * ep)
    ccc = (c[0] * (gg - 1.0) * eg * (fs + pinf * gp))
    pg = (-bbb + np.sqrt(bbb * bbb + 4.0 * ccc)) * 0.5
    pp = pg + fs
    phig = (c[0] * (gg - 1.0) * eg) / pg
    phip = 1.0 - phig
    rog, rop = c[0] / phig, c[5] / phip
    tg = pg / (rog * rrg)
    tp = ((pp + pinf) * gp) / ((gp - 1.0) * rop * cpp)
    m = phig < emin
    phig = np.where(m, emin, phig)
    phip = np.where(m, 1.0 - phig, phip)
    ug, vg, wg, tg, pg = (np.where(m, a, b) for a, b in ((up, ug), (vp, vg), (wp, wg), (tp, tg), (pp, pg)))
    m = phip < emin
    phip = np.where(m, emin, phip)
    phig = np.where(m, 1.0 - phip, phig)
    up, vp, wp, tp, pp = (np.where(m, a, b) for a, b in ((ug, up), (vg, vp), (wg, wp), (tg, tp), (pg, pp)))
    m = (phig >= emin) & (phig <= emax)
    psig = (phig - emin) / (emax - emin)
    f = -(psig * psig * (2.0 * psig - 3.0))
    ug, vg, wg, tg, pg = (np.where(m, f * a + (1.0 - f) * b, a)
                          for a, b in ((ug, up), (vg, vp), (wg, wp), (tg, tp), (pg, pp)))
    m = (phip >= emin) & (phip <= emax)
    psig = (phip - emin) / (emax - emin)
    f = -(psig * psig * (2.0 * psig - 3.0))
    up, vp, wp, tp, pp = (np.where(m, f * a + (1.0 - f) * b, a)
                          for a, b in ((up, ug), (vp, vg), (wp, wg), (tp, tg), (pp, pg)))
    rog = pg / (rrg * tg)
    rop = (pp + pinf) * gp / ((gp - 1.0) * cpp * tp)
    return np.stack([ug, vg, wg, pg, pp, tg, up, vp, wp, phig, tp, rog, rop])


def test_es16_8_restatement():
    assert es16_8(123456.789) == "  1.23456789E+05"
    assert es16_8(-1.0e-300) == " -1.00000000-300"
    assert es16_8(0.0) == "  0.00000000E+00"
    assert es16_8(float("nan")) == "             NaN"


def test_write_tecplot_format(tmp_path):
    spec = cases.shock_bubble(n=3, alpha_min=0.1)
    m = spec.mesh
    rng = np.random.default_rng(4)
    fields = rng.standard_normal((13, m.neles)) * 10.0 ** rng.integers(-120, 120, (13, m.neles))
    fields[0, :3] = [0.0, np.nan, -np.inf]
    p = tmp_path / "t.dat"
    write_tecplot(str(p), m, fields)
    assert p.read_text() == expected_tecplot(m, fields)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_FP64_PARITY, PREC_MIXED])
def test_async_output_matches_synchronous(tmp_path, precision):
    spec = cases.shock_bubble(n=8, alpha_min=0.1)
    m = spec.mesh
    with Case(m, spec.params(precision=precision)) as a, Case(m, spec.params(precision=precision)) as b:
        for c in (a, b):
            c.set_state(0.0, spec.cu, spec.ghost_prims)
            c.step(5, diagnostics=False)
        t1 = a.output_async(str(tmp_path / "r_async.in"), str(tmp_path / "t_async.dat"), mesh=m)
        a.step(7, diagnostics=False)            # overlaps the copy and the writer
        t2 = a.output_async(str(tmp_path / "r_async2.in"))
        a.output_wait(t1)
        a.output_wait(t2)
        tb, cu, gp = b.state()                  # the state at the first snapshot
        dp = ctypes.POINTER(ctypes.c_double)
        cu_c, gp_c = np.ascontiguousarray(cu), np.ascontiguousarray(gp)
        assert lib().hp_write_restart(str(tmp_path / "r_sync.in").encode(), m.neles, m.nghosts, tb,
                                      cu_c.ctypes.data_as(dp), gp_c.ctypes.data_as(dp)) == 0
        b.step(7, diagnostics=False)
        _, cu2, _ = b.state()
        _, cu2a, _ = a.state()
    assert (tmp_path / "r_async.in").read_bytes() == (tmp_path / "r_sync.in").read_bytes()
    assert (tmp_path / "t_async.dat").read_text() == expected_tecplot(m, tecplot_fields(cu, spec.flow))
    np.testing.assert_array_equal(cu2a, cu2)   # output did not disturb the steps
    assert (tmp_path / "r_async2.in").stat().st_size > 0


@pytest.mark.gpu
def test_state_into_caller_buffers():
    """Case.state(out=...) fills caller buffers (e.g. pinned memory) with the
    same values as a fresh read-back."""
    spec = cases.shock_bubble(n=6, alpha_min=0.1)
    m = spec.mesh
    with Case(m, spec.params(precision=PREC_FP64_PARITY)) as c:
        c.set_state(0.0, spec.cu, spec.ghost_prims)
        c.step(3, diagnostics=False)
        t, cu, gp = c.state()
        bufs = (np.full(10 * m.neles, np.nan), np.full(6 * m.nghosts + 5, np.nan))
        t2, cu2, gp2 = c.state(out=bufs)
        with pytest.raises(ValueError):
            c.state(out=(np.zeros(3), bufs[1]))
    assert t2 == t
    np.testing.assert_array_equal(cu2, cu)
    np.testing.assert_array_equal(gp2, gp)
