"""Shared body of the no-allocation tests (tests/test_zz_no_alloc.py): runs
bf_cuda_fit_noalloc and bf_cuda_fit on the same device buffers and compares every
output bit for bit.

Imported by the tests in their own process, and run as a script in a fresh child
process whose first library call is the no-allocation entry point:

    python tests/noalloc_check.py      # prints BITWISE_EQUAL or MISMATCH [...]
"""

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

KEYS = ("params", "status", "iterations", "chi2", "cov", "se", "ustatus")


def _device_outputs(torch, n, p, dev):
    # Filled with -1 so that an output the kernels never write shows up as a mismatch.
    f32, i32 = torch.float32, torch.int32
    return {"params": torch.full((n, p), -1.0, dtype=f32, device=dev),
            "status": torch.full((n,), -1, dtype=i32, device=dev),
            "iterations": torch.full((n,), -1, dtype=i32, device=dev),
            "chi2": torch.full((n,), -1.0, dtype=f32, device=dev),
            "cov": torch.full((n, p, p), -1.0, dtype=f32, device=dev),
            "se": torch.full((n, p), -1.0, dtype=f32, device=dev),
            "ustatus": torch.full((n,), -1, dtype=i32, device=dev)}


def _outs(capi, o):
    return capi.FitOutputs(*(C.c_void_p(o[k].data_ptr()) for k in KEYS))


def _as_bytes(o):
    return {k: o[k].cpu().numpy().tobytes() for k in KEYS}


def compare(with_p0: bool, noalloc_first: bool) -> list:
    """Fits 20,000 pseudo-Voigt spectra (M=512, uncertainties) twice through
    bf_cuda_fit_noalloc and once through bf_cuda_fit on a context, on the same
    device buffers.  Returns the outputs that differ (empty: bitwise equal)."""
    import torch

    import batchfit_b200 as bf
    from batchfit_b200 import _capi
    from batchfit_b200 import workloads as W

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    w = W.pseudo_voigt_plain(n=20_000, seed=21)
    n, p = w.y.shape[0], 4
    x = torch.from_numpy(w.x).to(dev)
    y = torch.from_numpy(w.y).to(dev)
    p0 = None
    if with_p0:
        rng = np.random.default_rng(5)
        start = np.array([2.5, 0.0, 1.0, 0.5], np.float32) * rng.uniform(0.8, 1.2, (n, p)).astype(np.float32)
        p0 = torch.from_numpy(start).to(dev)
    opts = bf.solver_options(w.model, w.lower, w.upper, "parity")
    dp = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
    args = _capi.FitArgs(2, n, w.x.size, dp(x), dp(y), dp(p0), _capi.BF_MEMORY_DEVICE, 1, 0, opts)
    stream = torch.cuda.current_stream(dev)

    def noalloc_twice():
        # A call with N == 0 loads the module and the kernels and launches nothing.
        warm = _capi.FitArgs(2, 0, w.x.size, None, None, None, _capi.BF_MEMORY_DEVICE, 1, 0, opts)
        rc = lib.bf_cuda_fit_noalloc(C.byref(warm), C.byref(_outs(_capi, _device_outputs(torch, 1, p, dev))),
                                     C.c_void_p(stream.cuda_stream))
        assert rc == _capi.BF_OK, _capi.last_error()
        runs = []
        for _ in range(2):
            got = _device_outputs(torch, n, p, dev)
            torch.cuda.synchronize()
            rc = lib.bf_cuda_fit_noalloc(C.byref(args), C.byref(_outs(_capi, got)), C.c_void_p(stream.cuda_stream))
            assert rc == _capi.BF_OK, _capi.last_error()
            stream.synchronize()
            runs.append(_as_bytes(got))
        return runs

    def with_context():
        ref = _device_outputs(torch, n, p, dev)
        torch.cuda.synchronize()
        bf.context(0).fit(args, _outs(_capi, ref))
        return _as_bytes(ref)

    if noalloc_first:
        runs = noalloc_twice()
        ref = with_context()
    else:
        ref = with_context()
        runs = noalloc_twice()
    return [f"call {i}: {k}" for i, got in enumerate(runs) for k in KEYS if got[k] != ref[k]]


if __name__ == "__main__":
    bad = compare(False, True) + compare(True, True)
    print(f"MISMATCH {bad}" if bad else "BITWISE_EQUAL")
