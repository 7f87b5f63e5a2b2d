"""The header-only C++ API (include/batchfit_cuda.hpp), the twin of the reference's
Context / make_batch / fit_batch / submit_batch -> PendingBatch API
(include/batchfit/metal/batch.hpp:160-310): tests/cpp/twin_check.cpp is compiled
with g++ against the header and the built library and run.  Without a GPU it must
report the device unavailable with std::runtime_error; on the GPU its results must
equal the C ABI's bit for bit, with the reference's exception types."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "batchfit_b200")


def _compile(tmp_path):
    cxx = shutil.which("g++")
    assert cxx, "g++ is required to build the C++ API check"
    exe = str(tmp_path / "twin_check")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "twin_check.cpp"), "-L", LIB_DIR, "-lbatchfit_cuda",
           f"-Wl,-rpath,{LIB_DIR}", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    return exe


def test_cpp_api_compiles_and_reports_no_device(tmp_path):
    from batchfit_b200 import _capi

    exe = _compile(tmp_path)
    if _capi.load().bf_cuda_available():
        return  # the GPU test below runs the full check on this machine
    res = subprocess.run([exe, "cpu"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0 and "OK" in res.stdout, res.stdout + res.stderr


@pytest.mark.gpu
def test_cpp_api_matches_the_c_abi_on_the_gpu(bf, tmp_path):
    exe = _compile(tmp_path)
    res = subprocess.run([exe, "gpu"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and "OK" in res.stdout, res.stdout + res.stderr
