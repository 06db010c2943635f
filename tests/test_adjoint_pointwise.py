"""Hand-written reverse-mode pointwise functions of the adjoint (inviscid and
viscous flux Jacobian-transpose products) against dual-number forward mode
through the forward physics, compiled for the host CPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
def test_pointwise_reverse_mode_matches_dual_numbers(tmp_path):
    exe = str(tmp_path / "pointwise_adjoint")
    src = os.path.join(HERE, "native", "pointwise_adjoint.cu")
    subprocess.run([NVCC, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-x", "cu", "-o", exe,
                    src], check=True, capture_output=True, timeout=300)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "worst relative error" in r.stdout
