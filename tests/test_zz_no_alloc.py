"""bf_cuda_fit_noalloc: the fit entry point for callers that cannot allocate GPU
memory (a host whose memory pool already owns the device, a real-time pipeline
that forbids allocation while it runs, a callback that may only enqueue work on a
stream it was given).  Its scratch lives in a fixed static device array, so this
test checks, through the C ABI, that its results equal bf_cuda_fit's on the same
device buffers, on two calls in a row (the shared scratch is reused and its work
counter cleared), and that sizes beyond the array are rejected.

Named to be collected last: a run that stops at the first failure has already run
every other test.  It also passes alone in a fresh process."""

import ctypes as C

import numpy as np
import pytest

from batchfit_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_outputs(torch, n, p, dev):
    return {"params": torch.empty((n, p), dtype=torch.float32, device=dev),
            "status": torch.empty(n, dtype=torch.int32, device=dev),
            "iterations": torch.empty(n, dtype=torch.int32, device=dev),
            "chi2": torch.empty(n, dtype=torch.float32, device=dev),
            "cov": torch.empty((n, p, p), dtype=torch.float32, device=dev),
            "se": torch.empty((n, p), dtype=torch.float32, device=dev),
            "ustatus": torch.empty(n, dtype=torch.int32, device=dev)}


def _outs(capi, o):
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    return capi.FitOutputs(dp(o["params"]), dp(o["status"]), dp(o["iterations"]), dp(o["chi2"]), dp(o["cov"]),
                           dp(o["se"]), dp(o["ustatus"]))


def _as_numpy(o):
    return {k: v.cpu().numpy() for k, v in o.items()}


def _assert_same(a, b):
    # The tolerance of the fit parity tests; identical kernels give identical bits.
    for key in ("status", "iterations", "ustatus"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    for key in ("params", "chi2", "cov", "se"):
        np.testing.assert_allclose(a[key], b[key], rtol=2e-4, atol=2e-4, err_msg=key)


@pytest.mark.parametrize("with_p0", [False, True])
def test_noalloc_matches_fit_on_two_calls(bf, with_p0):
    import torch

    from batchfit_b200 import _capi

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    w = W.pseudo_voigt_plain(n=20_000, seed=21)
    n, p = w.y.shape[0], 4
    x = torch.from_numpy(w.x).to(dev)
    y = torch.from_numpy(w.y).to(dev)
    p0 = None
    if with_p0:
        guesses, _ = bf.guess(w.x, w.y, w.model)
        fallback = np.array([2, 0, 1.7, 0.5], np.float32)
        guesses[~np.isfinite(guesses).all(axis=1)] = fallback
        p0 = torch.from_numpy(guesses).to(dev)
    opts = bf.solver_options(w.model, w.lower, w.upper, "parity")
    dp = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
    args = _capi.FitArgs(2, n, w.x.size, dp(x), dp(y), dp(p0), _capi.BF_MEMORY_DEVICE, 1, 0, opts)

    # The existing entry point on the same device buffers.
    ref = _device_outputs(torch, n, p, dev)
    torch.cuda.synchronize()
    bf.context(0).fit(args, _outs(_capi, ref))
    ref = _as_numpy(ref)

    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        got = _device_outputs(torch, n, p, dev)
        torch.cuda.synchronize()
        rc = lib.bf_cuda_fit_noalloc(C.byref(args), C.byref(_outs(_capi, got)), C.c_void_p(stream.cuda_stream))
        assert rc == _capi.BF_OK, _capi.last_error()
        stream.synchronize()
        _assert_same(_as_numpy(got), ref)


def test_noalloc_rejects_sizes_beyond_its_scratch(bf):
    import torch

    from batchfit_b200 import _capi

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    m, n = 8, 262_129  # one more pseudo-Voigt fit than the 4 MiB scratch holds guesses for
    x = torch.linspace(-1, 1, m, device=dev)
    y = torch.zeros((n, m), device=dev)
    opts = bf.solver_options("pseudo_voigt", [-np.inf] * 4, [np.inf] * 4, "parity")
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    args = _capi.FitArgs(2, n, m, dp(x), dp(y), None, _capi.BF_MEMORY_DEVICE, 0, 0, opts)
    o = _device_outputs(torch, 1, 4, dev)
    rc = lib.bf_cuda_fit_noalloc(C.byref(args), C.byref(_outs(_capi, o)), None)
    assert rc == _capi.BF_ERR_INVALID_ARGUMENT
    assert "4 MiB" in _capi.last_error() and "262128" in _capi.last_error()
    host = _capi.FitArgs(2, 4, m, dp(x), dp(y), None, _capi.BF_MEMORY_HOST, 0, 0, opts)
    assert lib.bf_cuda_fit_noalloc(C.byref(host), C.byref(_outs(_capi, o)), None) == _capi.BF_ERR_INVALID_ARGUMENT
