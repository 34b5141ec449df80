"""The FP64 force kernels seed 1/sqrt(x) with the double-precision
approximate instruction and apply one third-order correction, whose error is
~(5/16)(2e)^3 for a seed error e: FP64-exact only while e < 2^-18.  This
measures e on the device (tests/cuda/rsqrt_seed_error.cu)."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
SRC = Path(__file__).resolve().parent / "cuda" / "rsqrt_seed_error.cu"


def test_seed_error_below_cubic_threshold(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "seed"
    subprocess.run([nvcc, "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    str(SRC), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    err = float(re.search(r": ([0-9.eE+-]+) \(2\^", out).group(1))
    print(out.strip())
    assert err < 2.0 ** -18, out
