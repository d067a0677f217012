"""The C++ drop-in headers (include/cusbf/*): compiled against the C ABI
library here, and run on the GPU with checks restating the reference's unit
tests (tests/cpp/test_cpp_api.cu)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "cusbf_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_api.cu")


def _build(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    if not os.path.exists(os.path.join(LIB_DIR, "libsbf_b200.so")):
        pytest.fail("libsbf_b200.so is not built")
    exe = str(tmp_path / "test_cpp_api")
    cmd = [nvcc, "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIB_DIR, "-lsbf_b200", "-Xlinker", "-rpath", "-Xlinker", LIB_DIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_cpp_headers_compile(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_cpp_api_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp api checks: ok" in r.stdout
