import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "multiphase-code_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

REFERENCE_DIR = os.environ.get("HYDRA_REFERENCE_DIR",
                               "/root/reference/HydraPhase_60_FPC_5mill")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def have_reference() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_DIR, "geometry_files", "grid_proc0000.dat"))


@pytest.fixture(scope="session")
def reference_dir():
    if not have_reference():
        pytest.skip("reference checkout not mounted")
    return REFERENCE_DIR
