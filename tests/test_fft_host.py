"""The spectral form's FFT templates run on the host (nvcc, no GPU): transform lengths against a
direct FP64 DFT and the 2-D tile correlation against FP64 direct sums."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "ampcor_b200", "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.skipif(not (os.path.exists(NVCC) or shutil.which("nvcc")), reason="nvcc not found")
def test_fft_templates_on_host(tmp_path):
    exe = str(tmp_path / "fft_host_check")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-arch=sm_100a", "-I", CSRC, "-o", exe,
                    os.path.join(HERE, "fft_host_check.cu")], check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
