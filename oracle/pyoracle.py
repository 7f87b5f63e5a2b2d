"""Test infrastructure only: ctypes access to the CPU checkers.

* ``port``  -- oracle/liboracle.so, the plain-C restatement of the reference
  batchfit CPU fitting path (solver.hpp, initial_guess.hpp, uncertainty.hpp).
* ``ref``   -- oracle/_ref/libbatchfit_ref.so, the reference's own C++ CPU path
  compiled from its sources by oracle/Makefile (absent when it was never built).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module.  The batchfit_b200 product never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libbatchfit_ref.so")

MODELS = {"gaussian": 0, "lorentzian": 1, "pseudo_voigt": 2, "two_lorentzian": 3}
PCOUNT = {0: 3, 1: 3, 2: 4, 3: 8, 100: 2, 101: 1, 102: 1}  # 100-102: the reference tests' Line, Constant, Exponential


class Options(C.Structure):
    """cpu::SolverOptions scalars (include/batchfit/cpu/solver.hpp:26-41)."""

    _fields_ = [
        ("set", C.c_uint32),
        ("max_iterations", C.c_uint32),
        ("initial_lambda", C.c_double),
        ("gradient_tolerance", C.c_double),
        ("step_tolerance", C.c_double),
        ("cost_tolerance", C.c_double),
        ("compensated_sum", C.c_uint32),
        ("scaled_cholesky", C.c_uint32),
    ]


class Counters(C.Structure):
    _fields_ = [("cost_passes", C.c_uint64), ("linearize_passes", C.c_uint64), ("iterations", C.c_uint64)]


def make_options(max_iterations=100, initial_lambda=1e-3, gradient_tolerance=None, step_tolerance=None,
                 cost_tolerance=None, compensated_sum=False, scaled_cholesky=False, dtype=np.float32):
    f32 = np.dtype(dtype) == np.float32
    o = Options()
    o.set = 1
    o.max_iterations = max_iterations
    o.initial_lambda = initial_lambda
    o.gradient_tolerance = (1e-5 if f32 else 1e-10) if gradient_tolerance is None else gradient_tolerance
    o.step_tolerance = (1e-6 if f32 else 1e-10) if step_tolerance is None else step_tolerance
    o.cost_tolerance = (1e-6 if f32 else 1e-12) if cost_tolerance is None else cost_tolerance
    o.compensated_sum = int(bool(compensated_sum))
    o.scaled_cholesky = int(bool(scaled_cholesky))
    return o


_port = None
_ref = None


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def load_port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            raise RuntimeError(f"oracle port not built: run `make -C {HERE}`")
        lib = C.CDLL(PORT_PATH)
        vp, sz, i32p, u32p = C.c_void_p, C.c_size_t, C.POINTER(C.c_int32), C.POINTER(C.c_uint32)
        for suffix in ("f32", "f64"):
            f = getattr(lib, f"bfo_fit_{suffix}")
            f.argtypes = [C.c_int, sz, sz, vp, vp, vp, vp, vp, C.POINTER(Options), C.c_int, vp, vp, vp, vp,
                          vp, vp, vp, C.POINTER(Counters)]
            f.restype = C.c_int
            g = getattr(lib, f"bfo_guess_{suffix}")
            g.argtypes = [C.c_int, sz, sz, vp, vp, vp, vp, vp]
            g.restype = C.c_int
            h = getattr(lib, f"bfo_cholesky_solve_{suffix}")
            h.argtypes = [C.c_uint, vp, vp, C.c_int]
            h.restype = C.c_int
            u = getattr(lib, f"bfo_uncertainty_{suffix}")
            real = C.c_float if suffix == "f32" else C.c_double
            u.argtypes = [C.c_int, sz, vp, vp, C.c_int32, real, vp, vp, vp, vp, vp]
            u.restype = C.c_int
            e = getattr(lib, f"bfo_eval_{suffix}")
            e.argtypes = [C.c_int, real, vp]
            e.restype = real
            j = getattr(lib, f"bfo_jacobian_{suffix}")
            j.argtypes = [C.c_int, real, vp, vp]
            j.restype = None
        lib.bfo_kahan_add_f32.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.bfo_kahan_add_f32.restype = None
        _port = lib
    return _port


def ref_available():
    return os.path.exists(REF_PATH)


def load_ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference build absent: run `make -C oracle ref REFERENCE=<batchfit tree>`")
        lib = C.CDLL(REF_PATH)
        vp, sz = C.c_void_p, C.c_size_t
        lib.bfref_fit.argtypes = [C.c_int, C.c_int, sz, sz, vp, vp, vp, vp, vp, C.POINTER(Options), C.c_int,
                                  C.c_uint, vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_double)]
        lib.bfref_fit.restype = C.c_int
        lib.bfref_guess.argtypes = [C.c_int, C.c_int, sz, sz, vp, vp, vp, vp, vp]
        lib.bfref_guess.restype = C.c_int
        lib.bfref_cholesky_solve.argtypes = [C.c_int, C.c_uint, vp, vp, C.c_int]
        lib.bfref_cholesky_solve.restype = C.c_int
        lib.bfref_last_error.restype = C.c_char_p
        lib.bfref_hardware_concurrency.restype = C.c_uint
        _ref = lib
    return _ref


@dataclass
class FitOutput:
    params: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    chi2: np.ndarray
    covariance: np.ndarray | None = None
    stderr: np.ndarray | None = None
    uncertainty_status: np.ndarray | None = None
    guess_seconds: float = 0.0
    fit_seconds: float = 0.0
    counters: Counters | None = None


def _prep(model, x, y, p0, lower, upper, dtype):
    mid = MODELS[model] if isinstance(model, str) else int(model)
    p = PCOUNT[mid]
    dtype = np.dtype(dtype)
    x = np.ascontiguousarray(x, dtype=dtype)
    y = np.ascontiguousarray(y, dtype=dtype)
    if y.ndim == 1:
        y = y.reshape(1, -1)
    n, m = y.shape
    assert x.shape == (m,)
    if p0 is not None:
        p0 = np.ascontiguousarray(np.broadcast_to(np.asarray(p0, dtype=dtype), (n, p)))
    lower = np.ascontiguousarray(np.broadcast_to(np.asarray(-np.inf if lower is None else lower, dtype=dtype), (p,)))
    upper = np.ascontiguousarray(np.broadcast_to(np.asarray(np.inf if upper is None else upper, dtype=dtype), (p,)))
    return mid, p, dtype, x, y, n, m, p0, lower, upper


def fit(impl, model, x, y, p0=None, lower=None, upper=None, dtype=np.float32, options=None,
        uncertainties=False, workers=None, count_passes=False):
    """Run the reference fitting path ("ref") or its restatement ("port")."""
    mid, p, dtype, x, y, n, m, p0, lower, upper = _prep(model, x, y, p0, lower, upper, dtype)
    out = FitOutput(np.empty((n, p), dtype), np.empty(n, np.int32), np.empty(n, np.uint32), np.empty(n, dtype))
    if uncertainties:
        out.covariance = np.empty((n, p, p), dtype)
        out.stderr = np.empty((n, p), dtype)
        out.uncertainty_status = np.empty(n, np.int32)
    opt = C.byref(options) if options is not None else None
    if impl == "port":
        lib = load_port()
        fn = lib.bfo_fit_f32 if dtype == np.float32 else lib.bfo_fit_f64
        counters = Counters()
        rc = fn(mid, n, m, _ptr(x), _ptr(y), _ptr(p0), _ptr(lower), _ptr(upper), opt, int(uncertainties),
                _ptr(out.params), _ptr(out.status), _ptr(out.iterations), _ptr(out.chi2), _ptr(out.covariance),
                _ptr(out.stderr), _ptr(out.uncertainty_status), C.byref(counters) if count_passes else None)
        if rc:
            raise RuntimeError(f"oracle port failed ({rc})")
        out.counters = counters if count_passes else None
    elif impl == "ref":
        lib = load_ref()
        seconds = (C.c_double * 2)()
        w = workers if workers else lib.bfref_hardware_concurrency()
        rc = lib.bfref_fit(mid, dtype.itemsize, n, m, _ptr(x), _ptr(y), _ptr(p0), _ptr(lower), _ptr(upper), opt,
                           int(uncertainties), w, _ptr(out.params), _ptr(out.status), _ptr(out.iterations),
                           _ptr(out.chi2), _ptr(out.covariance), _ptr(out.stderr), _ptr(out.uncertainty_status),
                           seconds)
        if rc:
            raise RuntimeError(f"reference fit failed: {lib.bfref_last_error().decode()}")
        out.guess_seconds, out.fit_seconds = seconds[0], seconds[1]
    else:
        raise ValueError(impl)
    return out


def guess(impl, model, x, y, dtype=np.float32):
    """initial_guess<T,Model> per row -> (params[N,P], guess_status[N], baseline[N])."""
    mid, p, dtype, x, y, n, m, _, _, _ = _prep(model, x, y, None, None, None, dtype)
    params = np.empty((n, p), dtype)
    status = np.empty(n, np.int32)
    baseline = np.empty(n, dtype)
    if impl == "port":
        lib = load_port()
        fn = lib.bfo_guess_f32 if dtype == np.float32 else lib.bfo_guess_f64
        rc = fn(mid, n, m, _ptr(x), _ptr(y), _ptr(params), _ptr(status), _ptr(baseline))
    else:
        rc = load_ref().bfref_guess(mid, dtype.itemsize, n, m, _ptr(x), _ptr(y), _ptr(params), _ptr(status),
                                    _ptr(baseline))
    if rc:
        raise RuntimeError(f"guess failed ({rc})")
    return params, status, baseline


def cholesky_solve(impl, matrix, rhs, scaled=False, dtype=np.float64):
    a = np.ascontiguousarray(matrix, dtype=dtype).copy()
    b = np.ascontiguousarray(rhs, dtype=dtype).copy()
    p = b.shape[0]
    if impl == "port":
        lib = load_port()
        fn = lib.bfo_cholesky_solve_f32 if np.dtype(dtype) == np.float32 else lib.bfo_cholesky_solve_f64
        ok = fn(p, _ptr(a), _ptr(b), int(scaled))
    else:
        ok = load_ref().bfref_cholesky_solve(np.dtype(dtype).itemsize, p, _ptr(a), _ptr(b), int(scaled))
    return bool(ok == 1), a, b


def uncertainty(model, x, params, fit_status, chi2, lower, upper, dtype=np.float64):
    """estimate_uncertainty<T,Model> for one accepted state (port)."""
    mid = MODELS[model] if isinstance(model, str) else int(model)
    p = PCOUNT[mid]
    dtype = np.dtype(dtype)
    x = np.ascontiguousarray(x, dtype=dtype)
    params = np.ascontiguousarray(params, dtype=dtype)
    lower = np.ascontiguousarray(np.broadcast_to(np.asarray(lower, dtype=dtype), (p,)))
    upper = np.ascontiguousarray(np.broadcast_to(np.asarray(upper, dtype=dtype), (p,)))
    cov = np.empty((p, p), dtype)
    se = np.empty(p, dtype)
    us = C.c_int32()
    lib = load_port()
    fn = lib.bfo_uncertainty_f32 if dtype == np.float32 else lib.bfo_uncertainty_f64
    fn(mid, x.shape[0], _ptr(x), _ptr(params), int(fit_status), float(chi2), _ptr(lower), _ptr(upper), _ptr(cov),
       _ptr(se), C.byref(us))
    return cov, se, int(us.value)


def eval_model(model, x, params, dtype=np.float64):
    mid = MODELS[model] if isinstance(model, str) else int(model)
    lib = load_port()
    params = np.ascontiguousarray(params, dtype=dtype)
    fn = lib.bfo_eval_f32 if np.dtype(dtype) == np.float32 else lib.bfo_eval_f64
    return np.array([fn(mid, float(v), _ptr(params)) for v in np.atleast_1d(x)], dtype=dtype)


def jacobian(model, x, params, dtype=np.float64):
    mid = MODELS[model] if isinstance(model, str) else int(model)
    p = PCOUNT[mid]
    lib = load_port()
    params = np.ascontiguousarray(params, dtype=dtype)
    fn = lib.bfo_jacobian_f32 if np.dtype(dtype) == np.float32 else lib.bfo_jacobian_f64
    out = np.empty(p, dtype)
    fn(mid, float(x), _ptr(params), _ptr(out))
    return out


def kahan_add_f32(terms, start=0.0):
    lib = load_port()
    s, c = C.c_float(start), C.c_float(0.0)
    for t in terms:
        lib.bfo_kahan_add_f32(float(t), C.byref(s), C.byref(c))
    return s.value
