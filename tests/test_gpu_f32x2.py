"""The paired FP32 instructions of the FFT butterflies
(gpunufft_b200/csrc/f32x2.cuh: add.rn / sub.rn / mul.rn / fma.rn .f32x2)
give, lane for lane, the bits of the scalar round-to-nearest operations
(tests/cxx/f32x2_check.cu, 4 M results incl. signed zeros, infinities, NaN
and subnormals), so replacing the scalar code changed no result."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

pytestmark = pytest.mark.gpu


def test_paired_fp32_equals_scalar_bitwise(tmp_path):
    exe = str(tmp_path / "f32x2_check")
    cmd = [os.path.join(CUDA, "bin", "nvcc"), "-std=c++17", "-O2",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "gpunufft_b200", "csrc"),
           os.path.join(ROOT, "tests", "cxx", "f32x2_check.cu"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln.split() for ln in r.stdout.splitlines()]
    assert ["failures", "0"] in lines
