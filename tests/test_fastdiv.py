"""The multiply-shift divider of the transform passes (FastDiv in
gpunufft_b200/csrc/fftcore.cuh, host-callable) against integer division
on the CPU: tests/cxx/fastdiv_check.cu, compiled with nvcc for sm_100a,
runs its host code only."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_fastdiv_equals_integer_division(tmp_path):
    exe = str(tmp_path / "fastdiv_check")
    cmd = [os.path.join(CUDA, "bin", "nvcc"), "-std=c++17", "-O2",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "gpunufft_b200", "csrc"),
           os.path.join(ROOT, "tests", "cxx", "fastdiv_check.cu"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    lines = [ln.split() for ln in r.stdout.splitlines()]
    assert ["failures", "0"] in lines
    assert int([ln for ln in lines if ln[0] == "checks"][0][1]) > 3_000_000
