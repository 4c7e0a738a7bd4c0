"""The device reciprocal used by the flux formulas (vt::recip_nr, a hardware
estimate refined by two Newton-Raphson steps) against CUDA's IEEE division
1.0 / x: at most one unit in the last place apart, on 2.4 million inputs."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_newton_reciprocal_matches_division(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "gpu_reciprocal_check")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    "-I", os.path.join(ROOT, "vortex-transport_b200", "csrc"),
                    os.path.join(ROOT, "tests", "gpu_reciprocal_check.cu"), "-o", exe],
                   check=True, capture_output=True, text=True, timeout=600)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    m = re.search(r"samples (\d+) max_ulp (\d+) differing (\d+)", out)
    assert m, out
    samples, max_ulp, differing = (int(g) for g in m.groups())
    assert samples == 148 * 256 * 64
    assert max_ulp <= 1, out
    print(out.strip())
