"""Compile the extraction helpers of kc_kernels.cuh for the host and check
window extraction, canonical form and bucket-only routing against a
from-definition reference for every k in 1..64 (CPU only)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not available")
def test_extraction_helpers(tmp_path):
    exe = tmp_path / "helpers_test"
    subprocess.check_call([NVCC, "-std=c++20", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                           os.path.join(ROOT, "tests", "native", "helpers_test.cu"), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")
