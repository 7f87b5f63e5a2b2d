"""bf_cuda_fit_noalloc: the fit entry point for callers that cannot allocate GPU
memory (a host whose memory pool already owns the device, a real-time pipeline
that forbids allocation while it runs, a callback that may only enqueue work on a
stream it was given).  Its scratch lives in a fixed static device array, so these
tests check, through the C ABI, that its results equal bf_cuda_fit's on the same
device buffers bit for bit (both launch the same kernels with the same lanes per
fit), on two calls in a row (the shared scratch is reused and its work counter
cleared), and that sizes beyond the array and non-float32 y are rejected.

The comparison runs in this process, after whatever ran before it, and in a fresh
child process whose first library call is the no-allocation entry point (no
bf_cuda_context exists there when it runs).  The shared body is
tests/noalloc_check.py.

Named to be collected last: a run that stops at the first failure has already run
every other test."""

import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import noalloc_check  # noqa: E402


@pytest.mark.parametrize("with_p0", [False, True])
def test_noalloc_matches_fit_bitwise_on_two_calls(bf, with_p0):
    assert noalloc_check.compare(with_p0, noalloc_first=False) == []


def test_noalloc_first_call_in_a_fresh_process(bf):
    res = subprocess.run([sys.executable, os.path.join(HERE, "noalloc_check.py")], capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert "BITWISE_EQUAL" in res.stdout, res.stdout[-2000:]


def test_noalloc_rejects_sizes_beyond_its_scratch_and_half_y(bf):
    import torch

    from batchfit_b200 import _capi

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    m, n = 8, 262_129  # one more pseudo-Voigt fit than the 4 MiB scratch holds guesses for
    x = torch.linspace(-1, 1, m, device=dev)
    y = torch.zeros((n, m), device=dev)
    opts = bf.solver_options("pseudo_voigt", [-np.inf] * 4, [np.inf] * 4, "parity")
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    bufs = [torch.empty(16, dtype=torch.float32, device=dev) for _ in range(7)]
    outs = _capi.FitOutputs(*(dp(b) for b in bufs))
    args = _capi.FitArgs(2, n, m, dp(x), dp(y), None, _capi.BF_MEMORY_DEVICE, 0, 0, opts)
    assert lib.bf_cuda_fit_noalloc(C.byref(args), C.byref(outs), None) == _capi.BF_ERR_INVALID_ARGUMENT
    assert "4 MiB" in _capi.last_error() and "262128" in _capi.last_error()
    host = _capi.FitArgs(2, 4, m, dp(x), dp(y), None, _capi.BF_MEMORY_HOST, 0, 0, opts)
    assert lib.bf_cuda_fit_noalloc(C.byref(host), C.byref(outs), None) == _capi.BF_ERR_INVALID_ARGUMENT
    half = _capi.FitArgs(2, 4, m, dp(x), dp(y), None, _capi.BF_MEMORY_DEVICE, 0, 0, opts, _capi.BF_Y_FLOAT16)
    assert lib.bf_cuda_fit_noalloc(C.byref(half), C.byref(outs), None) == _capi.BF_ERR_INVALID_ARGUMENT
    assert "float32" in _capi.last_error()
