"""Extract small golden fixtures from the reference's own shipped outputs.

Run in a container where the reference checkout is mounted:
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/HydraPhase_60_FPC_5mill")
