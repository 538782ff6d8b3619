"""Drop-in boundary checks that need no GPU: the C ABI exports everything
include/hydraphase.h declares, the reference-format readers/writers agree
with the oracle's independent readers, and argument errors come back as
HP_E_* codes (the reference prints and STOPs instead,
src/mod_Fluxmodule.F90:15-16)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, have_reference, REFERENCE_DIR
from hydraphase import (HP_E_ARG, HP_E_CUDA, HP_E_IO, HP_E_UNSUPPORTED, Case, HydraError, LIB_PATH,
                        MeshArrays, cases, lib, make_params, read_flow, read_mesh, read_restart,
                        write_restart)
from hydraphase._lib import EXPORTED_SYMBOLS, HpMesh, HpParams


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "hydraphase.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(hp_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    declared = _declared_symbols()
    assert len(declared) >= 18
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(hp_\w+)", out.stdout))
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert set(EXPORTED_SYMBOLS) <= exported
    L = lib()
    for s in declared:
        assert hasattr(L, s)


def test_flow_reader_matches_oracle_parser(tmp_path):
    spec = cases.shock_bubble(n=3)
    cases.write_case_dir(spec, str(tmp_path))
    p = read_flow(str(tmp_path / "flow.in"))
    ref = O.parse_flow_in(open(tmp_path / "flow.in").read())
    for k, v in ref.items():
        assert getattr(p, k) == v, k


@pytest.mark.skipif(not have_reference(), reason="reference checkout not mounted")
def test_shipped_flow_and_mesh(reference_dir):
    p = read_flow(os.path.join(reference_dir, "flow.in"))
    ref = O.parse_flow_in(open(os.path.join(reference_dir, "flow.in")).read())
    for k, v in ref.items():
        assert getattr(p, k) == v, k
    assert (p.myflux, p.myorder, p.niter, p.itersub) == (2, 2, 2, 5)
    m = read_mesh(reference_dir)
    _, om = O.read_case_dir(reference_dir)
    np.testing.assert_array_equal(m.x, om.x)
    np.testing.assert_array_equal(m.y, om.y)
    np.testing.assert_array_equal(m.z, om.z)
    np.testing.assert_array_equal(m.elem, om.elem)
    np.testing.assert_array_equal(m.ghost, om.ghost)


def test_shipped_mesh_through_reference_format(tmp_path):
    """The shipped mesh (committed fixture), written back in the reference's
    grid/bc text layout with 17 significant digits as its list-directed
    output has them, and read by the library's reader: identical arrays.
    Runs without the reference checkout."""
    from conftest import shipped_case
    flow, om = shipped_case()
    g = tmp_path / "geometry_files"
    g.mkdir()
    (tmp_path / "flow.in").write_text(str(np.load(os.path.join(ROOT, "tests", "golden",
                                                               "shipped_mesh.npz"))["flow_in"]))
    with open(g / "grid_proc0000.dat", "w") as f:
        f.write(f"{om.nodes:12d}{om.neles:12d}\n")
        nd = np.column_stack([np.arange(1, om.nodes + 1), om.x, om.y, om.z, om.gid, om.gid])
        np.savetxt(f, nd, fmt="%12d %25.16E %25.16E %25.16E %16d %11d")
        np.savetxt(f, np.column_stack([np.arange(1, om.neles + 1), om.elem]), fmt="%12d")
    with open(g / "bc_proc0000.in", "w") as f:
        f.write(f"{om.nghosts:12d}\n")
        np.savetxt(f, om.ghost, fmt="%12d")
    (g / "proc_bc0000.in").write_text("           0           0\n")
    p = read_flow(str(tmp_path / "flow.in"))
    assert (p.myflux, p.myorder, p.niter, p.itersub) == (2, 2, 2, 5)
    # the dispersed-phase groups the five-phase model reads (flow.in lines
    # after myorder, as, ts)
    assert (p.rhoq, p.rhor, p.rhos) == (2500.0, 1950.0, 2700.0)
    assert (p.radq, p.radr, p.rads) == (5.0e-6, 20.0e-6, 7.50e-6)
    assert (p.phiqinit, p.phirinit, p.phisinit) == (0.4600, 0.1550, 0.1180)
    assert flow["rhoq"] == p.rhoq and flow["phisinit"] == p.phisinit
    m = read_mesh(str(tmp_path))
    for k in ("x", "y", "z", "elem", "ghost"):
        np.testing.assert_array_equal(getattr(m, k), getattr(om, k), err_msg=k)


@pytest.mark.skipif(not have_reference(), reason="reference checkout not mounted")
def test_shipped_restart_reader(reference_dir):
    m = read_mesh(reference_dir)
    t, cu, gp = read_restart(os.path.join(reference_dir, "restart_files", "restart0000.in"), m.neles, m.nghosts)
    t2, cu2, gp2 = O.read_restart(os.path.join(reference_dir, "restart_files", "restart0000.in"),
                                  m.neles, m.nghosts)
    assert t == t2
    np.testing.assert_array_equal(cu.ravel(), cu2)
    np.testing.assert_array_equal(gp, gp2)


def test_case_dir_round_trip(tmp_path):
    spec = cases.shock_bubble(n=4, alpha_min=0.1)
    cases.write_case_dir(spec, str(tmp_path))
    m = read_mesh(str(tmp_path))
    np.testing.assert_array_equal(m.elem, spec.mesh.elem)
    np.testing.assert_array_equal(m.ghost, spec.mesh.ghost)
    np.testing.assert_array_equal(m.x, spec.mesh.x)
    np.testing.assert_array_equal(m.z, spec.mesh.z)
    t, cu, gp = read_restart(str(tmp_path / "restart_files" / "restart0000.in"), m.neles, m.nghosts)
    np.testing.assert_array_equal(cu, spec.cu)
    np.testing.assert_array_equal(gp, spec.ghost_prims)
    # NaN entries survive a write/read cycle (the shipped restart holds some)
    cu2 = spec.cu.copy()
    cu2[:, 3] = np.nan
    write_restart(str(tmp_path / "r.in"), 1.5e-6, cu2, gp)
    t3, cu3, _ = read_restart(str(tmp_path / "r.in"), m.neles, m.nghosts)
    assert t3 == 1.5e-6
    np.testing.assert_array_equal(cu3, cu2)


def test_reader_errors(tmp_path):
    with pytest.raises(HydraError) as e:
        read_flow(str(tmp_path / "missing.in"))
    assert e.value.code == HP_E_IO
    with pytest.raises(HydraError) as e:
        read_mesh(str(tmp_path))
    assert e.value.code == HP_E_IO
    (tmp_path / "flow.in").write_text("# empty\n1.0 2.0\n")
    with pytest.raises(HydraError) as e:
        read_flow(str(tmp_path / "flow.in"))
    assert e.value.code == HP_E_IO


def _tiny():
    return cases.shock_bubble(n=2)


def test_create_rejects_bad_meshes():
    spec = _tiny()
    m = spec.mesh
    bad = m.elem.copy()
    bad[0, 0] = m.nodes + 5                      # node id out of range
    with pytest.raises(HydraError) as e:
        Case(MeshArrays(m.x, m.y, m.z, bad, m.ghost), spec.params())
    assert e.value.code == HP_E_ARG and "node id" in str(e.value)
    bad = m.elem.copy()
    bad[1, 5] = 0                                # neighbour id out of range
    with pytest.raises(HydraError) as e:
        Case(MeshArrays(m.x, m.y, m.z, bad, m.ghost), spec.params())
    assert e.value.code == HP_E_ARG
    gh = m.ghost.copy()
    gh[0, 3] = 7                                 # face side must be 1..4
    with pytest.raises(HydraError) as e:
        Case(MeshArrays(m.x, m.y, m.z, m.elem, gh), spec.params())
    assert e.value.code == HP_E_ARG
    for bad_flux in (0, 4):                      # no such flux (the reference stops)
        with pytest.raises(HydraError) as e:
            Case(m, spec.params(myflux=bad_flux))
        assert e.value.code == HP_E_ARG and "myflux" in str(e.value)
    with pytest.raises(HydraError) as e:
        Case(m, spec.params(face_mode=4))
    assert e.value.code == HP_E_ARG and "face_mode" in str(e.value)
    with pytest.raises(HydraError) as e:
        Case(m, spec.params(wall_fp64_layers=-1))
    assert e.value.code == HP_E_ARG and "wall_fp64_layers" in str(e.value)


def test_partition_ghosts_unsupported():
    spec = _tiny()
    m = spec.mesh
    keep = [np.ascontiguousarray(a) for a in (m.x, m.y, m.z)] + [np.ascontiguousarray(m.elem, np.int32),
                                                                   np.ascontiguousarray(m.ghost, np.int32)]
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    hm = HpMesh(m.nodes, m.neles, m.nghosts, 3, dp(keep[0]), dp(keep[1]), dp(keep[2]), ip(keep[3]), ip(keep[4]))
    h = ctypes.c_void_p()
    p = spec.params()
    rc = lib().hp_create(ctypes.byref(hm), ctypes.byref(p), ctypes.byref(h))
    assert rc == HP_E_UNSUPPORTED
    assert b"partition" in lib().hp_create_error()


def test_no_gpu_fails_loudly():
    """On a machine without a CUDA device the engine refuses to run instead of
    falling back to a CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    spec = _tiny()
    with pytest.raises(HydraError) as e:
        Case(spec.mesh, spec.params())
    assert e.value.code == HP_E_CUDA


def test_params_layout_matches_header(tmp_path):
    """hp_params is shared by C callers, the Python mirror and Fortran bind(C)
    interfaces: the C compiler's size and every field offset equal the
    mirror's."""
    assert HpParams.cfl.offset == 29 * 8
    assert HpParams.face_mode.offset == 296
    names = [f[0] for f in HpParams._fields_]
    cname = {"as_": "as"}
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"hydraphase.h\"\nint main(void) {\n"
                   "  printf(\"%zu\\n\", sizeof(hp_params));\n" +
                   "".join(f'  printf("%zu\\n", offsetof(hp_params, {cname.get(n, n)}));\n' for n in names) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(HpParams)
    assert vals[1:] == [getattr(HpParams, n).offset for n in names]


def test_host_thread_share():
    """hp_set_host_threads sets the calling thread's set-up threads (0 = one
    per core) and rejects a negative count; no GPU needed."""
    from hydraphase import HP_E_ARG, lib
    assert lib().hp_set_host_threads(2) == 0
    assert lib().hp_set_host_threads(0) == 0
    assert lib().hp_set_host_threads(-1) == HP_E_ARG


def test_partition_constants_match_header():
    """The Python mirror's halo iblank codes and exchange points are the
    header's enums."""
    from hydraphase._lib import HP_IBLANK_HALO1, HP_IBLANK_HALO2, HP_X_DT, HP_X_HALO
    hdr = open(os.path.join(ROOT, "include", "hydraphase.h")).read()
    vals = {k: int(v) for k, v in re.findall(r"\b(HP_IBLANK_HALO[12]|HP_X_DT|HP_X_HALO)\s*=\s*(\d+)", hdr)}
    assert vals == {"HP_IBLANK_HALO1": HP_IBLANK_HALO1, "HP_IBLANK_HALO2": HP_IBLANK_HALO2,
                    "HP_X_DT": HP_X_DT, "HP_X_HALO": HP_X_HALO}
