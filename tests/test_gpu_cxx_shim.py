"""The C++ drop-in (include/gpuNUFFT_operator_factory.hpp and
include/gpuNUFFT_operator.hpp, header-only over the C ABI): a C++ caller
written against the upstream's GpuNUFFTOperatorFactory / GpuNUFFTOperator
signatures (tests/cxx/gpunufft_cxx_test.cpp) builds against include/ and
libgpunufft_b200.so, and on the GPU reproduces the upstream operators'
outputs for the upstream gtest case it restates (forward 2D_32_32_4, all
eight factory flag combinations) within 1e-5, besides its own checks
(upstream FFT-stage known answers, coil-combined channels, device arrays
equal host arrays, precomputed operators equal the original, errors as
exceptions)."""
import os
import subprocess

import numpy as np
import pytest

from tests.golden.make_golden import known_cases
from tests.helpers import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "gpunufft_cxx_test.cpp")
LIBDIR = os.path.join(ROOT, "gpunufft_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
FIXTURE = os.path.join(ROOT, "tests", "golden", "upstream_gpu_known.npz")


def _build(tmp_path):
    exe = str(tmp_path / "gpunufft_cxx_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), SRC, "-o", exe,
           "-L" + LIBDIR, "-lgpunufft_b200",
           "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-Wl,-rpath," + os.path.join(CUDA,
                                                                "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cxx_shim_builds_against_the_library(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run(["ldd", exe], capture_output=True, text=True)
    assert "libgpunufft_b200.so" in r.stdout


@pytest.mark.gpu
def test_cxx_shim_runs_upstream_gtest_cases(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln.split() for ln in r.stdout.splitlines()]
    assert ["failures", "0"] in lines
    gold = np.load(FIXTURE)
    case = known_cases()["fwd_2d_32_4"]
    fwd = [ln for ln in lines if ln[0] == "forward_2d_32_32_4"]
    assert len(fwd) == 8
    for ln in fwd:
        op_type, n = int(ln[1]), int(ln[2])
        vals = np.array(ln[3:], np.float64).reshape(n, 2)
        y = vals[:, 0] + 1j * vals[:, 1]
        tex, bal = op_type in (1, 3), op_type in (2, 3)
        key = f"fwd_2d_32_4/{int(tex)}{int(bal)}"
        idx = gold[key + "/idx"]
        assert np.array_equal(idx, np.arange(n)) and n == len(case[11])
        assert rel_l2(y[idx], gold[key + "/val"]) < 1e-5
    b1 = [ln for ln in lines if ln[0] == "deapo_2d_b1"][0]
    up = gold["deapo_2d_b1/01/val"][0]
    assert abs(float(b1[1]) - up.real) < 1e-5 * abs(up)
