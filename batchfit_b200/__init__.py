"""batchfit B200 backend: batched bounded Levenberg-Marquardt spectral fitting on
NVIDIA B200 (sm_100a).

``fit`` mirrors the reference Python API (python/batchfit/__init__.py:63-112):
shared x[M], fit-major y[N,M], p0 [P] / [N,P] / None (data-only guesses on the
GPU), bounds (lower, upper) as scalars or [P] (equal bounds fix a coordinate), and
the same FitResult / FitResultWithUncertainties tuples, FitStatus and
UncertaintyStatus codes.  Like the reference's explicit GPU device, results are
float32 and an explicit CUDA request never falls back to the CPU.

Inputs may be numpy arrays (host memory; the library pipelines the copies) or CUDA
tensors exposing ``__cuda_array_interface__`` (device memory, zero copy; outputs
are then torch CUDA tensors).
"""

from __future__ import annotations

import ctypes as C
import threading
from enum import IntEnum
from typing import NamedTuple

import numpy as np

from . import _capi

__version__ = "0.1.0"
__all__ = ["fit", "fit_batch", "fit_npy", "fit_physical", "autotune", "Server", "FitResult", "FitResultWithUncertainties", "FitStatus",
           "UncertaintyStatus", "cuda_available", "MODELS", "__version__"]

MODELS = {"gaussian": 0, "lorentzian": 1, "pseudo_voigt": 2, "two_lorentzian": 3}
_PARAMETERS = {"gaussian": 3, "lorentzian": 3, "pseudo_voigt": 4, "two_lorentzian": 8}
_POLICIES = {"reference": _capi.BF_POLICY_REFERENCE, "parity": _capi.BF_POLICY_PARITY}


class FitStatus(IntEnum):
    converged = 0
    max_iterations = 1
    singular_matrix = 2
    invalid_input = 3
    degenerate_data = 4
    unresolved_peak = 5


class UncertaintyStatus(IntEnum):
    available = 0
    not_converged = 1
    insufficient_dof = 2
    singular_matrix = 3
    active_bound = 4
    invalid_input = 5


class FitResult(NamedTuple):
    params: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    chi2: np.ndarray


class FitResultWithUncertainties(NamedTuple):
    params: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    chi2: np.ndarray
    covariance: np.ndarray
    stderr: np.ndarray
    uncertainty_status: np.ndarray


_contexts: dict[int, _capi.Context] = {}
_contexts_lock = threading.Lock()


def context(device: int = 0) -> _capi.Context:
    """The process-wide context of a CUDA device (created on first use)."""
    with _contexts_lock:
        ctx = _contexts.get(device)
        if ctx is None:
            ctx = _capi.Context(device)
            _contexts[device] = ctx
        return ctx


def cuda_available() -> bool:
    """Whether the library loads and an sm_100-class device is present."""
    return bool(_capi.load().bf_cuda_available())


def _real_array(value, name):
    array = np.asarray(value)
    if array.dtype.kind not in "fiu":
        raise TypeError(f"{name} must contain real numeric values")
    return array


def _is_device(value) -> bool:
    return hasattr(value, "__cuda_array_interface__")


def solver_options(model: str, bounds_lower, bounds_upper, policy: str = "parity", **overrides):
    """bf_solver_options for `model`: the policy's defaults, the given bounds, and
    any field overrides (max_iterations, initial_lambda, gradient_tolerance,
    step_tolerance, cost_tolerance, scaled_cholesky, noise_floor, step_quantum)."""
    if policy not in _POLICIES:
        raise ValueError(f"policy must be one of {tuple(_POLICIES)}")
    o = _capi.default_options(MODELS[model], _POLICIES[policy])
    p = _PARAMETERS[model]
    for k in range(p):
        o.lower[k] = float(bounds_lower[k])
        o.upper[k] = float(bounds_upper[k])
    for key, value in overrides.items():
        if not hasattr(o, key):
            raise ValueError(f"unknown solver option {key!r}")
        setattr(o, key, value)
    return o


def _bounds(bounds, p):
    if bounds is None:
        return np.full(p, -np.inf, np.float32), np.full(p, np.inf, np.float32)
    if not isinstance(bounds, (tuple, list)) or len(bounds) != 2:
        raise ValueError("bounds must be (lower, upper), each scalar or [P]")
    lower, upper = (_real_array(value, "bounds") for value in bounds)
    if lower.shape not in ((), (p,)) or upper.shape not in ((), (p,)):
        raise ValueError(f"each bound must be scalar or have shape [{p}]")
    maximum = np.finfo(np.float32).max
    if any(np.any(np.isfinite(b) & (np.abs(b.astype(np.float64)) > maximum)) for b in (lower, upper)):
        raise ValueError("finite bounds must be representable in the fitting dtype")
    lower = np.ascontiguousarray(np.broadcast_to(lower, (p,)), dtype=np.float32)
    upper = np.ascontiguousarray(np.broadcast_to(upper, (p,)), dtype=np.float32)
    # python/bindings.cpp:264-273 rejects these before fitting.
    if (np.any(np.isnan(lower)) or np.any(np.isnan(upper)) or np.any(lower > upper)
            or np.any(lower == np.inf) or np.any(upper == -np.inf)):
        raise ValueError("invalid parameter bounds")
    return lower, upper


def fit(x, y, model="lorentzian", p0=None, bounds=None, device="auto", *, uncertainties=False,
        policy="parity", group_lanes=0, options=None):
    """Fit shared x[M] and y[N,M]; return params[N,P], status/iterations/chi2[N].

    A single y[M] is accepted as N=1.  ``device`` is "auto" or "cuda"; both run on
    the GPU and never fall back.  ``policy`` selects the stopping rules: "parity"
    (default) iterates to the float32 noise floor to match the float64 solution,
    "reference" uses the reference float solver's tolerances.  ``options`` may be
    a ready bf_solver_options (see ``solver_options``) and then overrides both.
    """
    if model not in _PARAMETERS:
        raise ValueError(f"unknown model {model!r}; choose one of {tuple(_PARAMETERS)}")
    if device not in ("auto", "cuda"):
        raise ValueError("device must be 'auto' or 'cuda' (the CPU and Metal devices belong to the reference package)")
    if not isinstance(uncertainties, (bool, np.bool_)):
        raise TypeError("uncertainties must be a boolean")
    if _is_device(x) or _is_device(y):
        return _fit_device(x, y, model, p0, bounds, bool(uncertainties), policy, group_lanes, options)
    x, y = _real_array(x, "x"), _real_array(y, "y")
    if x.ndim != 1 or not x.size:
        raise ValueError("x must have nonempty shape [M]")
    if y.ndim == 1:
        y = y.reshape(1, -1)
    if y.ndim != 2 or y.shape[1] != x.size:
        raise ValueError("y must have shape [N,M] matching x[M]")
    x = np.ascontiguousarray(x, dtype=np.float32)
    # float16 y is the opt-in half-precision storage (half the copy bytes); the
    # values are fitted exactly as given, converted to float32 on the GPU.
    y_format = _capi.BF_Y_FLOAT16 if y.dtype == np.float16 else _capi.BF_Y_FLOAT32
    y = np.ascontiguousarray(y, dtype=np.float16 if y_format == _capi.BF_Y_FLOAT16 else np.float32)
    n, p = y.shape[0], _PARAMETERS[model]
    if p0 is not None:
        p0 = _real_array(p0, "p0")
        if p0.shape == (p,):
            p0 = np.broadcast_to(p0, (n, p))
        if p0.shape != (n, p):
            raise ValueError(f"p0 must have shape [{p}] or [{n},{p}]")
        p0 = np.ascontiguousarray(p0, dtype=np.float32)
    lower, upper = _bounds(bounds, p)
    opts = options if options is not None else solver_options(model, lower, upper, policy)
    ctx = context(0)
    params = np.empty((n, p), np.float32)
    status = np.empty(n, np.int32)
    iterations = np.empty(n, np.uint32)
    chi2 = np.empty(n, np.float32)
    cov = np.empty((n, p, p), np.float32) if uncertainties else None
    se = np.empty((n, p), np.float32) if uncertainties else None
    us = np.empty(n, np.int32) if uncertainties else None
    ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
    args = _capi.FitArgs(MODELS[model], n, x.size, ptr(x), ptr(y), ptr(p0), _capi.BF_MEMORY_HOST,
                         int(bool(uncertainties)), int(group_lanes), opts, y_format)
    outs = _capi.FitOutputs(ptr(params), ptr(status), ptr(iterations), ptr(chi2), ptr(cov), ptr(se), ptr(us))
    ctx.fit(args, outs)
    if uncertainties:
        return FitResultWithUncertainties(params, status, iterations, chi2, cov, se, us)
    return FitResult(params, status, iterations, chi2)


def _device_segment(x, y, model, p0, bounds, uncertainties, policy, group_lanes, options, half_ok=False):
    """Validate torch CUDA inputs and allocate outputs -> (FitArgs, FitOutputs, result, keep-alive)."""
    import torch  # device-memory inputs come from torch (plumbing only)

    if not (isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor)):
        raise TypeError("device inputs must be torch CUDA tensors")
    if x.dtype != torch.float32 or y.dtype not in (torch.float32,) + ((torch.float16,) if half_ok else ()):
        raise TypeError("device inputs must be float32" + (" (y may be float16)" if half_ok else ""))
    if y.dim() == 1:
        y = y.reshape(1, -1)
    if x.dim() != 1 or x.numel() == 0 or y.dim() != 2 or y.shape[1] != x.numel():
        raise ValueError("expected x[M] and y[N,M] with M>0")
    if x.device != y.device:
        raise ValueError("x and y must be on the same device")
    x = x.contiguous()
    y = y.contiguous()
    n, p = y.shape[0], _PARAMETERS[model]
    if p0 is not None:
        p0 = torch.as_tensor(p0, dtype=torch.float32, device=y.device)
        if p0.shape == (p,):
            p0 = p0.expand(n, p)
        if tuple(p0.shape) != (n, p):
            raise ValueError(f"p0 must have shape [{p}] or [{n},{p}]")
        p0 = p0.contiguous()
    lower, upper = _bounds(bounds, p)
    opts = options if options is not None else solver_options(model, lower, upper, policy)
    kw = dict(device=y.device)
    params = torch.empty((n, p), dtype=torch.float32, **kw)
    status = torch.empty(n, dtype=torch.int32, **kw)
    iterations = torch.empty(n, dtype=torch.int32, **kw)
    chi2 = torch.empty(n, dtype=torch.float32, **kw)
    cov = torch.empty((n, p, p), dtype=torch.float32, **kw) if uncertainties else None
    se = torch.empty((n, p), dtype=torch.float32, **kw) if uncertainties else None
    us = torch.empty(n, dtype=torch.int32, **kw) if uncertainties else None
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
    y_format = _capi.BF_Y_FLOAT16 if y.dtype == torch.float16 else _capi.BF_Y_FLOAT32
    args = _capi.FitArgs(MODELS[model], n, x.numel(), ptr(x), ptr(y), ptr(p0), _capi.BF_MEMORY_DEVICE,
                         int(uncertainties), int(group_lanes), opts, y_format)
    outs = _capi.FitOutputs(ptr(params), ptr(status), ptr(iterations), ptr(chi2), ptr(cov), ptr(se), ptr(us))
    if uncertainties:
        result = FitResultWithUncertainties(params, status, iterations, chi2, cov, se, us)
    else:
        result = FitResult(params, status, iterations, chi2)
    return args, outs, result, (x, y, p0)


def _fit_device(x, y, model, p0, bounds, uncertainties, policy, group_lanes, options):
    import torch

    args, outs, result, keep = _device_segment(x, y, model, p0, bounds, uncertainties, policy, group_lanes, options,
                                               half_ok=True)
    device = keep[1].device
    torch.cuda.current_stream(device).synchronize()
    context(device.index or 0).fit(args, outs)
    return result


def fit_batch(requests, *, fixed_mapping=False, graph=True):
    """Fit many independent requests of different models and M as one mixed batch.

    Each request is a dict with the arguments of ``fit``: ``x``, ``y``, and
    optionally ``model``, ``p0``, ``bounds``, ``uncertainties``, ``policy``,
    ``group_lanes`` and ``options``.  x/y may be numpy arrays (copied to the GPU)
    or torch CUDA tensors.  Returns one result per request, in order, as torch CUDA
    tensors.  All requests run in one persistent launch per kernel; each result is
    the one ``fit`` gives for the same request alone with the same lanes per fit.
    ``fixed_mapping`` runs every fit on one warp in request order (the plain
    mapping); ``graph=False`` launches the kernels one by one.
    """
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("CUDA fitting is unavailable: no CUDA device")
    segments, results, keep = [], [], []
    device = None
    for i, req in enumerate(requests):
        req = dict(req)
        model = req.pop("model", "lorentzian")
        if model not in _PARAMETERS:
            raise ValueError(f"request {i}: unknown model {model!r}")
        x, y = req.pop("x"), req.pop("y")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        if not _is_device(x):
            x = torch.as_tensor(np.ascontiguousarray(_real_array(x, "x"), dtype=np.float32)).to(dev)
        if not _is_device(y):
            y = torch.as_tensor(np.ascontiguousarray(_real_array(y, "y"), dtype=np.float32)).to(dev)
        device = device or y.device
        p0 = req.pop("p0", None)
        unc = req.pop("uncertainties", False)
        if not isinstance(unc, (bool, np.bool_)):
            raise TypeError(f"request {i}: uncertainties must be a boolean")
        args, outs, result, k = _device_segment(x, y, model, p0, req.pop("bounds", None), bool(unc),
                                                req.pop("policy", "parity"), req.pop("group_lanes", 0),
                                                req.pop("options", None))
        if req:
            raise TypeError(f"request {i}: unexpected keys {sorted(req)}")
        segments.append(_capi.BatchSegment(args, outs))
        results.append(result)
        keep.append(k)
    if not segments:
        return []
    torch.cuda.current_stream(device).synchronize()
    flags = (_capi.BF_BATCH_FIXED_MAPPING if fixed_mapping else 0) | (0 if graph else _capi.BF_BATCH_NO_GRAPH)
    context(device.index or 0).fit_batch(segments, flags)
    return results


class _Ticket:
    """One submitted request: ``done()``, ``result()`` (blocks), ``latency_ms``."""

    def __init__(self, server, ticket, result, keep):
        self._server, self._ticket, self._result, self._keep = server, ticket, result, keep
        self._code = None
        self.latency_ms = None

    def done(self) -> bool:
        if self._code is not None:
            return True
        rc = self._server._lib.bf_server_poll(self._server._ptr, self._ticket)
        if rc < 0:
            _capi.check(-rc, "bf_server_poll")
        return rc == 1

    def cancel(self) -> bool:
        """Cancel the request if it has not been admitted yet (then ``result()``
        raises concurrent.futures.CancelledError); False once it is admitted."""
        if self._code is not None:
            return False
        rc = self._server._lib.bf_server_cancel(self._server._ptr, self._ticket)
        if rc < 0:
            _capi.check(-rc, "bf_server_cancel")
        return rc == 1

    def result(self):
        if self._code is None:
            latency = C.c_double()
            self._code = self._server._lib.bf_server_wait(self._server._ptr, self._ticket, C.byref(latency))
            self.latency_ms = latency.value
            self._server._live.pop(self._ticket, None)
        _capi.check(self._code, "server request")
        return self._result


class Server:
    """Continuous-batching fit server on one GPU (native scheduler thread).

    ``submit`` takes the arguments of ``fit`` (host arrays) and returns a ticket at
    once; requests are admitted while their device buffers fit ``memory_budget``
    bytes (0: 150 GB, capped by free memory), coalesced into mixed batches, and up
    to two batches run at once.  ``max_batch_fits`` caps the fits of one launch.
    """

    def __init__(self, device=0, memory_budget=0, max_batch_fits=0, fixed_mapping=False, graph=True,
                 max_in_flight=2):
        self._lib = _capi.load()
        self._ptr = C.c_void_p()
        flags = (_capi.BF_BATCH_FIXED_MAPPING if fixed_mapping else 0) | (0 if graph else _capi.BF_BATCH_NO_GRAPH)
        opt = _capi.ServerOptions(int(memory_budget), int(max_batch_fits), flags, int(max_in_flight))
        _capi.check(self._lib.bf_server_create(device, C.byref(opt), C.byref(self._ptr)), "bf_server_create")
        # Host buffers of every request that has not been collected: the scheduler
        # reads the inputs at admission and writes the outputs at completion.
        self._live = {}

    def submit(self, x, y, model="lorentzian", p0=None, bounds=None, *, uncertainties=False, policy="parity",
               options=None):
        if model not in _PARAMETERS:
            raise ValueError(f"unknown model {model!r}; choose one of {tuple(_PARAMETERS)}")
        if not isinstance(uncertainties, (bool, np.bool_)):
            raise TypeError("uncertainties must be a boolean")
        x = np.ascontiguousarray(_real_array(x, "x"), dtype=np.float32)
        y = np.ascontiguousarray(_real_array(y, "y"), dtype=np.float32)
        if y.ndim == 1:
            y = y.reshape(1, -1)
        if x.ndim != 1 or not x.size or y.ndim != 2 or y.shape[1] != x.size:
            raise ValueError("expected x[M] and y[N,M] with M>0")
        n, p = y.shape[0], _PARAMETERS[model]
        if p0 is not None:
            p0 = _real_array(p0, "p0")
            if p0.shape == (p,):
                p0 = np.broadcast_to(p0, (n, p))
            if p0.shape != (n, p):
                raise ValueError(f"p0 must have shape [{p}] or [{n},{p}]")
            p0 = np.ascontiguousarray(p0, dtype=np.float32)
        lower, upper = _bounds(bounds, p)
        opts = options if options is not None else solver_options(model, lower, upper, policy)
        params = np.empty((n, p), np.float32)
        status = np.empty(n, np.int32)
        iterations = np.empty(n, np.uint32)
        chi2 = np.empty(n, np.float32)
        cov = np.empty((n, p, p), np.float32) if uncertainties else None
        se = np.empty((n, p), np.float32) if uncertainties else None
        us = np.empty(n, np.int32) if uncertainties else None
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        args = _capi.FitArgs(MODELS[model], n, x.size, ptr(x), ptr(y), ptr(p0), _capi.BF_MEMORY_HOST,
                             int(bool(uncertainties)), 0, opts)
        outs = _capi.FitOutputs(ptr(params), ptr(status), ptr(iterations), ptr(chi2), ptr(cov), ptr(se), ptr(us))
        ticket = C.c_uint64()
        _capi.check(self._lib.bf_server_submit(self._ptr, C.byref(args), C.byref(outs), C.byref(ticket)),
                    "bf_server_submit")
        if uncertainties:
            result = FitResultWithUncertainties(params, status, iterations, chi2, cov, se, us)
        else:
            result = FitResult(params, status, iterations, chi2)
        self._live[ticket.value] = (x, y, p0, result)
        return _Ticket(self, ticket.value, result, None)

    def _fail_allocations(self, count: int):
        """Failure injection for tests: the next `count` admissions fail as if the
        device allocation ran out of memory (on the host; no GPU fault)."""
        _capi.check(self._lib.bf_server_fail_allocations(self._ptr, int(count)), "bf_server_fail_allocations")

    def stats(self) -> dict:
        st = _capi.ServerStats()
        _capi.check(self._lib.bf_server_get_stats(self._ptr, C.byref(st)), "bf_server_get_stats")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self):
        """Complete every submitted request, then release the server."""
        if self._ptr:
            self._lib.bf_server_destroy(self._ptr)
            self._ptr = C.c_void_p()
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(device: int = 0):
    """Time the LM kernel per (model, M bucket) at 8/16/32 lanes per fit on the
    device and keep the fastest for later mixed batches; returns lanes[4][8]."""
    t = context(device).autotune()
    return [[t.lanes[m][b] for b in range(8)] for m in range(4)]


def guess(x, y, model="lorentzian"):
    """Data-only initial guesses on the GPU -> (params[N,P], guess_status[N])."""
    if model not in _PARAMETERS:
        raise ValueError(f"unknown model {model!r}")
    x = np.ascontiguousarray(_real_array(x, "x"), dtype=np.float32)
    y = np.ascontiguousarray(_real_array(y, "y"), dtype=np.float32)
    if y.ndim == 1:
        y = y.reshape(1, -1)
    n, p = y.shape[0], _PARAMETERS[model]
    params = np.empty((n, p), np.float32)
    status = np.empty(n, np.int32)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    context(0).guess(MODELS[model], n, x.size, ptr(x), ptr(y), _capi.BF_MEMORY_HOST, ptr(params), ptr(status))
    return params, status


def fit_npy(*args, **kwargs):
    """Out-of-core fits from .npy files; see ``batchfit_b200.npy.fit_npy``."""
    from .npy import fit_npy as _fit_npy

    return _fit_npy(*args, **kwargs)


def fit_physical(x, y, model="lorentzian", p0=None, bounds=None, *, uncertainties=False, policy="parity",
                 group_lanes=0, options=None):
    """Fit float64 data in normalised coordinates, results in physical units.

    The reference's ``Coordinates`` recipe (include/batchfit/coordinates.hpp):
    x is centred and scaled by its half range, each spectrum by its largest |y|,
    in double on the GPU; the fit runs in float32 on the normalised data and
    parameters, chi2, covariance and standard errors come back in physical units
    as float64 numpy arrays.  ``p0`` is in physical units; ``bounds`` are in
    fitted (normalised) units, as the reference requires.
    """
    import torch

    if model not in _PARAMETERS:
        raise ValueError(f"unknown model {model!r}; choose one of {tuple(_PARAMETERS)}")
    x = np.ascontiguousarray(_real_array(x, "x"), dtype=np.float64)
    y = np.ascontiguousarray(_real_array(y, "y"), dtype=np.float64)
    if y.ndim == 1:
        y = y.reshape(1, -1)
    if x.ndim != 1 or not x.size or y.ndim != 2 or y.shape[1] != x.size:
        raise ValueError("expected x[M] and y[N,M] with M>0")
    n, p = y.shape[0], _PARAMETERS[model]
    if p0 is not None:
        p0 = np.asarray(_real_array(p0, "p0"), dtype=np.float64)
        if p0.shape == (p,):
            p0 = np.broadcast_to(p0, (n, p))
        if p0.shape != (n, p):
            raise ValueError(f"p0 must have shape [{p}] or [{n},{p}]")
        p0 = np.ascontiguousarray(p0)
    lower, upper = _bounds(bounds, p)
    opts = options if options is not None else solver_options(model, lower, upper, policy)
    dev = torch.device("cuda", torch.cuda.current_device())
    xd, yd = torch.from_numpy(x).to(dev), torch.from_numpy(y).to(dev)
    pd = None if p0 is None else torch.from_numpy(p0).to(dev)
    kw = dict(device=dev)
    params = torch.empty((n, p), dtype=torch.float64, **kw)
    status = torch.empty(n, dtype=torch.int32, **kw)
    iterations = torch.empty(n, dtype=torch.int32, **kw)
    chi2 = torch.empty(n, dtype=torch.float64, **kw)
    cov = torch.empty((n, p, p), dtype=torch.float64, **kw) if uncertainties else None
    se = torch.empty((n, p), dtype=torch.float64, **kw) if uncertainties else None
    us = torch.empty(n, dtype=torch.int32, **kw) if uncertainties else None
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
    args = _capi.PhysicalArgs(MODELS[model], n, x.size, ptr(xd), ptr(yd), ptr(pd), int(bool(uncertainties)),
                              int(group_lanes), opts)
    outs = _capi.PhysicalOutputs(ptr(params), ptr(status), ptr(iterations), ptr(chi2), ptr(cov), ptr(se), ptr(us))
    torch.cuda.current_stream(dev).synchronize()
    ctx = context(dev.index or 0)
    _capi.check(ctx._lib.bf_cuda_fit_physical(ctx.handle, C.byref(args), C.byref(outs)), "bf_cuda_fit_physical")
    np_ = lambda t: None if t is None else t.cpu().numpy()  # noqa: E731
    if uncertainties:
        return FitResultWithUncertainties(np_(params), np_(status), np_(iterations).astype(np.uint32), np_(chi2),
                                          np_(cov), np_(se), np_(us))
    return FitResult(np_(params), np_(status), np_(iterations).astype(np.uint32), np_(chi2))
