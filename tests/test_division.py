"""The fast correctly rounded FP64 division of the kernels (Markstein's
correction with a shared reciprocal, mdiv/mrcp in csrc/hp_kernels.cuh) must
equal the hardware IEEE quotient bit for bit whenever it does not flag its
operands.  tests/division_check.cu is compiled with nvcc and run on about
2.4e9 seeded random operand pairs (no flags expected in that range)."""
import os
import re
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_fast_division_equals_ieee(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "division_check")
    subprocess.run([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false",
                    "-o", exe, os.path.join(HERE, "division_check.cu")], check=True, capture_output=True)
    out = subprocess.run([exe, "2"], capture_output=True, text=True, timeout=300)
    m = re.search(r"pairs (\d+) flagged (\d+) mismatches (\d+)", out.stdout)
    assert m, out.stdout + out.stderr
    pairs, flagged, mism = map(int, m.groups())
    assert out.returncode == 0 and mism == 0, out.stdout
    assert pairs > 2_000_000_000 and flagged < pairs // 1000
