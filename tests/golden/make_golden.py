"""Extract small golden fixtures from the reference's own shipped outputs.

Run where the reference checkout is mounted, naming its project directory
on the command line or in HYDRA_REFERENCE_DIR:
    python tests/golden/make_golden.py /path/to/HydraPhase_60_FPC_5mill

Writes tests/golden/shipped_case.npz with
  velocity      Velocity.dat lines 131-140: (time, |u_g(cell 1)|) for the 10
                steps of flow.in (niter*itersub = 2*5), 17 significant digits
  restart_time  first record of restart_files/restart0000.in
  nan_cells     1-based element ids whose conserved state is NaN in the
                golden restart (the overset block that the merged mesh
                corrupts, see inputfiles/mergefiles.f90:100-110)
  sample_ids    1-based ids of a deterministic sample of finite cells
  sample_cu     cu(sample_ids, 1:10) from the golden restart
  ghost_ids     0-based ghost-list positions of a sample of ghosts
  ghost_prims   (ug, vg, wg, pg, tg, rog) at those ghosts from the restart
  var_sums      per-variable sums of cu over all finite cells

and tests/golden/shipped_mesh.npz, the shipped run's inputs, so that the run
can be repeated (by the oracle and on the GPU) without the reference:
  x, y, z       node coordinates of geometry_files/grid_proc0000.dat
  gid           the grid-id column of its node lines
  elem_delta    its element rows (nod1..4, nc1..4, iblank), each row stored
                as its difference from the previous row (int32; the merged
                structured blocks make these differences small and repetitive,
                so the file compresses to a few hundred kB)
  ghost_delta   the rows of geometry_files/bc_proc0000.in, coded the same way
  flow_in       the text of flow.in
  itter_in      the text of itter.in
proc_bc0000.in declares no partition ghosts; the loader checks that.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    vel = np.loadtxt(os.path.join(ref, "Velocity.dat")).reshape(-1, 2)[-10:]
    with open(os.path.join(ref, "geometry_files", "grid_proc0000.dat")) as f:
        nodes, neles = (int(t) for t in f.readline().split()[:2])
    with open(os.path.join(ref, "geometry_files", "bc_proc0000.in")) as f:
        nghosts = int(f.readline().split()[0])
    toks = open(os.path.join(ref, "restart_files", "restart0000.in")).read().split()
    vals = np.array(toks[: 1 + 10 * neles + 6 * nghosts], dtype=np.float64)
    t = float(vals[0])
    cu = vals[1:1 + 10 * neles].reshape(10, neles)
    gp = vals[1 + 10 * neles:].reshape(6, nghosts)
    nan_cells = np.where(np.isnan(cu).any(axis=0))[0] + 1
    finite = np.where(~np.isnan(cu).any(axis=0))[0]
    rng = np.random.default_rng(12345)
    sample = np.sort(rng.choice(finite, size=3000, replace=False))
    sample = np.unique(np.concatenate([[0], sample]))          # always cell 1
    gfin = np.where(~np.isnan(gp).any(axis=0))[0]
    gsample = np.sort(rng.choice(gfin, size=1000, replace=False))
    np.savez_compressed(
        os.path.join(HERE, "shipped_case.npz"),
        velocity=vel, restart_time=np.float64(t), nan_cells=nan_cells.astype(np.int32),
        sample_ids=(sample + 1).astype(np.int32), sample_cu=cu[:, sample].T.copy(),
        ghost_ids=gsample.astype(np.int32), ghost_prims=gp[:, gsample].T.copy(),
        var_sums=np.nansum(np.where(np.isnan(cu), 0.0, cu), axis=1),
        nodes=np.int32(nodes), neles=np.int32(neles), nghosts=np.int32(nghosts))
    print("wrote", os.path.join(HERE, "shipped_case.npz"), "nan cells:", nan_cells.size)
    write_mesh(ref)


def _delta(rows: np.ndarray) -> np.ndarray:
    r = rows.astype(np.int64)
    return np.diff(np.concatenate([np.zeros((1, r.shape[1]), np.int64), r]), axis=0).astype(np.int32)


def write_mesh(ref: str) -> None:
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    import oracle as O
    _, mesh = O.read_case_dir(ref)
    with open(os.path.join(ref, "geometry_files", "proc_bc0000.in")) as f:
        assert int(f.readline().split()[0]) == 0
    out = os.path.join(HERE, "shipped_mesh.npz")
    np.savez_compressed(
        out, x=mesh.x, y=mesh.y, z=mesh.z, gid=mesh.gid.astype(np.int32),
        elem_delta=_delta(mesh.elem), ghost_delta=_delta(mesh.ghost),
        flow_in=np.array(open(os.path.join(ref, "flow.in")).read()),
        itter_in=np.array(open(os.path.join(ref, "itter.in")).read()))
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HYDRA_REFERENCE_DIR", "")
    if not ref:
        raise SystemExit("usage: make_golden.py REFERENCE_PROJECT_DIR (or set HYDRA_REFERENCE_DIR)")
    main(ref)
