"""ctypes binding of the C ABI declared in include/batchfit_cuda.h.

Loads the in-tree batchfit_b200/libbatchfit_cuda.so.  There is no fallback: when
the library is missing, loading raises RuntimeError naming the build command.
"""

from __future__ import annotations

import concurrent.futures
import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# BATCHFIT_CUDA_LIBRARY may name another build of the same ABI (e.g. a debug build).
LIB_PATH = os.environ.get("BATCHFIT_CUDA_LIBRARY") or os.path.join(HERE, "libbatchfit_cuda.so")

BF_OK = 0
BF_ERR_INVALID_ARGUMENT = 1
BF_ERR_CUDA = 2
BF_ERR_UNAVAILABLE = 3
BF_ERR_BUSY = 4
BF_ERR_CANCELLED = 5
BF_MEMORY_HOST = 0
BF_MEMORY_DEVICE = 1
BF_POLICY_REFERENCE = 0
BF_POLICY_PARITY = 1

# Every entry point the header declares (checked by the CPU test suite).
EXPORTS = (
    "bf_cuda_last_error", "bf_cuda_available", "bf_cuda_version", "bf_cuda_context_create",
    "bf_cuda_context_destroy", "bf_cuda_default_options", "bf_cuda_fit", "bf_cuda_submit", "bf_cuda_ready",
    "bf_cuda_wait", "bf_cuda_guess", "bf_cuda_last_timing", "bf_cuda_host_alloc", "bf_cuda_host_free",
    "bf_cuda_max_points", "bf_cuda_measure_peaks", "bf_cuda_fit_noalloc", "bf_cuda_fit_batch",
    "bf_cuda_batch_max_points", "bf_cuda_autotune", "bf_cuda_get_tuning", "bf_cuda_set_tuning",
    "bf_server_create", "bf_server_destroy", "bf_server_submit", "bf_server_poll", "bf_server_wait",
    "bf_server_get_stats", "bf_server_cancel", "bf_server_fail_allocations", "bf_cuda_fit_npy", "bf_npy_inspect",
    "bf_cuda_fit_physical",
)

BF_Y_FLOAT32, BF_Y_FLOAT16 = 0, 1
BF_BATCH_FIXED_MAPPING = 1
BF_BATCH_NO_GRAPH = 2


class SolverOptions(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_uint32),
        ("initial_lambda", C.c_double),
        ("gradient_tolerance", C.c_double),
        ("step_tolerance", C.c_double),
        ("cost_tolerance", C.c_double),
        ("compensated_sum", C.c_uint32),
        ("scaled_cholesky", C.c_uint32),
        ("policy", C.c_uint32),
        ("noise_floor", C.c_double),
        ("step_quantum", C.c_double),
        ("lower", C.c_float * 8),
        ("upper", C.c_float * 8),
    ]


class FitArgs(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("n", C.c_uint64),
        ("m", C.c_uint32),
        ("x", C.c_void_p),
        ("y", C.c_void_p),
        ("p0", C.c_void_p),
        ("memory", C.c_int32),
        ("uncertainties", C.c_int32),
        ("group_lanes", C.c_int32),
        ("options", SolverOptions),
        ("y_format", C.c_int32),
    ]


class FitOutputs(C.Structure):
    _fields_ = [
        ("params", C.c_void_p),
        ("status", C.c_void_p),
        ("iterations", C.c_void_p),
        ("chi2", C.c_void_p),
        ("covariance", C.c_void_p),
        ("standard_errors", C.c_void_p),
        ("uncertainty_status", C.c_void_p),
    ]


class Peaks(C.Structure):
    _fields_ = [("fp32_tflops", C.c_double), ("fp64_tflops", C.c_double), ("mufu_ex2_gops", C.c_double),
                ("mufu_rcp_gops", C.c_double)]


class Timing(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
        ("launches", C.c_uint32),
        ("group_lanes", C.c_int32),
        ("grid", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("guess_ms", C.c_double),
        ("lm_ms", C.c_double),
        ("covariance_ms", C.c_double),
        ("batches", C.c_uint32),
    ]


class BatchSegment(C.Structure):
    _fields_ = [("args", FitArgs), ("out", FitOutputs)]


class Tuning(C.Structure):
    _fields_ = [("lanes", (C.c_int32 * 8) * 4), ("lm_ms", ((C.c_double * 3) * 8) * 4), ("tuned", C.c_int32)]


class ServerOptions(C.Structure):
    _fields_ = [("memory_budget", C.c_uint64), ("max_batch_fits", C.c_uint64), ("batch_flags", C.c_uint32),
                ("max_in_flight", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("fits_completed", C.c_uint64), ("batches", C.c_uint64), ("memory_in_use", C.c_uint64),
                ("memory_peak", C.c_uint64), ("memory_budget", C.c_uint64), ("max_batch_requests", C.c_uint64),
                ("gpu_ms", C.c_double)]


class NpyOptions(C.Structure):
    _fields_ = [("model", C.c_int32), ("uncertainties", C.c_int32), ("chunk_fits", C.c_uint64),
                ("in_flight", C.c_uint32), ("solver", SolverOptions)]


class NpyStats(C.Structure):
    _fields_ = [("fits", C.c_uint64), ("chunks", C.c_uint64), ("chunk_fits", C.c_uint64),
                ("wall_seconds", C.c_double), ("read_seconds", C.c_double), ("fit_seconds", C.c_double),
                ("write_seconds", C.c_double)]


class PhysicalArgs(C.Structure):
    _fields_ = [("model", C.c_int32), ("n", C.c_uint64), ("m", C.c_uint32), ("x", C.c_void_p), ("y", C.c_void_p),
                ("p0", C.c_void_p), ("uncertainties", C.c_int32), ("group_lanes", C.c_int32),
                ("options", SolverOptions)]


class PhysicalOutputs(C.Structure):
    _fields_ = [("params", C.c_void_p), ("status", C.c_void_p), ("iterations", C.c_void_p), ("chi2", C.c_void_p),
                ("covariance", C.c_void_p), ("standard_errors", C.c_void_p), ("uncertainty_status", C.c_void_p)]


_lib = None
_lock = threading.Lock()


def load():
    """Load the CUDA library (no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"batchfit CUDA library missing at {LIB_PATH}; build it with "
                               "`python -m batchfit_b200.build`")
        lib = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        lib.bf_cuda_last_error.restype = C.c_char_p
        lib.bf_cuda_available.restype = C.c_int
        lib.bf_cuda_version.restype = C.c_int
        lib.bf_cuda_context_create.argtypes = [C.c_int, C.POINTER(vp)]
        lib.bf_cuda_context_destroy.argtypes = [vp]
        lib.bf_cuda_context_destroy.restype = None
        lib.bf_cuda_default_options.argtypes = [C.c_int32, C.c_uint32, C.POINTER(SolverOptions)]
        lib.bf_cuda_fit.argtypes = [vp, C.POINTER(FitArgs), C.POINTER(FitOutputs)]
        lib.bf_cuda_submit.argtypes = [vp, C.POINTER(FitArgs), C.POINTER(FitOutputs), C.POINTER(vp)]
        lib.bf_cuda_ready.argtypes = [vp]
        lib.bf_cuda_wait.argtypes = [vp]
        lib.bf_cuda_guess.argtypes = [vp, C.c_int32, C.c_uint64, C.c_uint32, vp, vp, C.c_int32, vp, vp]
        lib.bf_cuda_last_timing.argtypes = [vp, C.POINTER(Timing)]
        lib.bf_cuda_host_alloc.argtypes = [C.c_size_t, C.POINTER(vp)]
        lib.bf_cuda_host_free.argtypes = [vp]
        lib.bf_cuda_max_points.argtypes = [C.c_int32]
        lib.bf_cuda_max_points.restype = C.c_uint32
        lib.bf_cuda_measure_peaks.argtypes = [vp, C.POINTER(Peaks)]
        lib.bf_cuda_fit_noalloc.argtypes = [C.POINTER(FitArgs), C.POINTER(FitOutputs), vp]
        lib.bf_cuda_fit_batch.argtypes = [vp, C.POINTER(BatchSegment), C.c_uint32, C.c_uint32]
        lib.bf_cuda_batch_max_points.restype = C.c_uint32
        lib.bf_cuda_autotune.argtypes = [vp, C.POINTER(Tuning)]
        lib.bf_cuda_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        lib.bf_cuda_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        lib.bf_server_create.argtypes = [C.c_int, C.POINTER(ServerOptions), C.POINTER(vp)]
        lib.bf_server_destroy.argtypes = [vp]
        lib.bf_server_destroy.restype = None
        lib.bf_server_submit.argtypes = [vp, C.POINTER(FitArgs), C.POINTER(FitOutputs), C.POINTER(C.c_uint64)]
        lib.bf_server_poll.argtypes = [vp, C.c_uint64]
        lib.bf_server_wait.argtypes = [vp, C.c_uint64, C.POINTER(C.c_double)]
        lib.bf_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
        lib.bf_server_cancel.argtypes = [vp, C.c_uint64]
        lib.bf_server_fail_allocations.argtypes = [vp, C.c_uint32]
        lib.bf_cuda_fit_npy.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(NpyOptions),
                                        C.POINTER(NpyStats)]
        lib.bf_cuda_fit_physical.argtypes = [vp, C.POINTER(PhysicalArgs), C.POINTER(PhysicalOutputs)]
        lib.bf_npy_inspect.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_uint64)]
        for name in EXPORTS:
            getattr(lib, name).restype = getattr(lib, name).restype or C.c_int
        _lib = lib
        return lib


def last_error() -> str:
    return load().bf_cuda_last_error().decode(errors="replace")


def check(rc: int, what: str = "batchfit CUDA call"):
    if rc == BF_OK:
        return
    message = last_error()
    if rc == BF_ERR_INVALID_ARGUMENT:
        raise ValueError(f"{what}: {message}")
    if rc == BF_ERR_UNAVAILABLE:
        raise RuntimeError(f"CUDA fitting is unavailable: {message}")
    if rc == BF_ERR_CANCELLED:
        raise concurrent.futures.CancelledError(f"{what}: {message}")
    raise RuntimeError(f"{what} failed ({rc}): {message}")


def default_options(model: int, policy: int = BF_POLICY_PARITY) -> SolverOptions:
    o = SolverOptions()
    check(load().bf_cuda_default_options(model, policy, C.byref(o)), "bf_cuda_default_options")
    return o


class Context:
    """One bf_cuda_context (owns streams and device staging buffers)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        self._ptr = C.c_void_p()
        check(self._lib.bf_cuda_context_create(device, C.byref(self._ptr)), "bf_cuda_context_create")

    @property
    def handle(self):
        return self._ptr

    def close(self):
        if self._ptr:
            self._lib.bf_cuda_context_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fit(self, args: FitArgs, outs: FitOutputs):
        check(self._lib.bf_cuda_fit(self._ptr, C.byref(args), C.byref(outs)), "bf_cuda_fit")

    def submit(self, args: FitArgs, outs: FitOutputs):
        pending = C.c_void_p()
        check(self._lib.bf_cuda_submit(self._ptr, C.byref(args), C.byref(outs), C.byref(pending)), "bf_cuda_submit")
        return pending

    def ready(self, pending) -> bool:
        rc = self._lib.bf_cuda_ready(pending)
        if rc < 0:
            check(-rc, "bf_cuda_ready")
        return rc == 1

    def wait(self, pending):
        check(self._lib.bf_cuda_wait(pending), "bf_cuda_wait")

    def guess(self, model, n, m, x_ptr, y_ptr, memory, params_ptr, status_ptr):
        check(self._lib.bf_cuda_guess(self._ptr, model, n, m, x_ptr, y_ptr, memory, params_ptr, status_ptr),
              "bf_cuda_guess")

    def measure_peaks(self) -> Peaks:
        p = Peaks()
        check(self._lib.bf_cuda_measure_peaks(self._ptr, C.byref(p)), "bf_cuda_measure_peaks")
        return p

    def fit_batch(self, segments, flags: int = 0):
        """Run a list of BatchSegment (device pointers) as one mixed batch."""
        arr = (BatchSegment * max(1, len(segments)))(*segments)
        check(self._lib.bf_cuda_fit_batch(self._ptr, arr, len(segments), flags), "bf_cuda_fit_batch")

    def autotune(self) -> Tuning:
        t = Tuning()
        check(self._lib.bf_cuda_autotune(self._ptr, C.byref(t)), "bf_cuda_autotune")
        return t

    def get_tuning(self) -> Tuning:
        t = Tuning()
        check(self._lib.bf_cuda_get_tuning(self._ptr, C.byref(t)), "bf_cuda_get_tuning")
        return t

    def set_tuning(self, t: Tuning):
        check(self._lib.bf_cuda_set_tuning(self._ptr, C.byref(t)), "bf_cuda_set_tuning")

    def timing(self) -> Timing:
        t = Timing()
        check(self._lib.bf_cuda_last_timing(self._ptr, C.byref(t)), "bf_cuda_last_timing")
        return t
