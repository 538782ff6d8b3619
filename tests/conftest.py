import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "multiphase-code_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

# The reference checkout is optional: tests that read its files directly run
# only when HYDRA_REFERENCE_DIR names its project directory.  The shipped run
# itself is available everywhere through tests/golden/shipped_mesh.npz.
REFERENCE_DIR = os.environ.get("HYDRA_REFERENCE_DIR", "")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def have_reference() -> bool:
    return bool(REFERENCE_DIR) and os.path.isfile(
        os.path.join(REFERENCE_DIR, "geometry_files", "grid_proc0000.dat"))


def shipped_case():
    """The reference's shipped run (merged overset mesh of 266,688 cells,
    its flow.in) from the committed fixture: (flow dict, oracle Mesh).
    The mesh rows are stored as row differences; see make_golden.py."""
    import numpy as np
    import oracle as O
    g = np.load(os.path.join(GOLDEN_DIR, "shipped_mesh.npz"))
    elem = np.cumsum(g["elem_delta"].astype(np.int64), axis=0).astype(np.int32)
    ghost = np.cumsum(g["ghost_delta"].astype(np.int64), axis=0).astype(np.int32)
    flow = O.parse_flow_in(str(g["flow_in"]))
    return flow, O.Mesh(g["x"], g["y"], g["z"], elem, ghost, g["gid"])


@pytest.fixture(scope="session")
def reference_dir():
    if not have_reference():
        pytest.skip("reference checkout not mounted")
    return REFERENCE_DIR
