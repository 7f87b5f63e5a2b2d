"""The C-ABI library loads, exports every entry point include/batchfit_cuda.h
declares, and validates arguments on the host.  No compute call is made here."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from batchfit_b200 import _capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "batchfit_cuda.h")


def declared_entry_points():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(bf_(?:cuda|server|npy)_\w+)\s*\(", text)))


def test_header_declares_the_binding_table():
    assert declared_entry_points() == sorted(_capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared_entry_points():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header():
    # bf_solver_options: 4 + 8*4 (after padding) + 3*4 + 8*2 + 2*8*4
    assert C.sizeof(_capi.SolverOptions) == 4 + 4 + 8 * 4 + 4 * 3 + 4 + 8 * 2 + 4 * 16
    assert C.sizeof(_capi.FitOutputs) == 7 * 8


@pytest.mark.parametrize("model", [0, 1, 2, 3])
def test_default_options(model):
    ref = _capi.default_options(model, _capi.BF_POLICY_REFERENCE)
    assert ref.max_iterations == 100 and ref.initial_lambda == 1e-3
    assert (ref.gradient_tolerance, ref.step_tolerance, ref.cost_tolerance) == (1e-5, 1e-6, 1e-6)
    par = _capi.default_options(model, _capi.BF_POLICY_PARITY)
    assert (par.gradient_tolerance, par.step_tolerance, par.cost_tolerance) == (1e-10, 1e-10, 1e-12)
    assert par.noise_floor == 16 and par.step_quantum == 16
    assert all(np.isinf(v) and v < 0 for v in par.lower) and all(np.isinf(v) and v > 0 for v in par.upper)


def test_invalid_default_options_rejected():
    lib = _capi.load()
    o = _capi.SolverOptions()
    assert lib.bf_cuda_default_options(7, 0, C.byref(o)) == _capi.BF_ERR_INVALID_ARGUMENT
    assert b"model" in lib.bf_cuda_last_error()
    assert lib.bf_cuda_default_options(0, 9, C.byref(o)) == _capi.BF_ERR_INVALID_ARGUMENT


def test_null_context_and_arguments_rejected():
    lib = _capi.load()
    args, outs = _capi.FitArgs(), _capi.FitOutputs()
    assert lib.bf_cuda_fit(None, C.byref(args), C.byref(outs)) == _capi.BF_ERR_INVALID_ARGUMENT
    pending = C.c_void_p()
    assert lib.bf_cuda_submit(None, C.byref(args), C.byref(outs), C.byref(pending)) == _capi.BF_ERR_INVALID_ARGUMENT
    assert lib.bf_cuda_wait(None) == _capi.BF_ERR_INVALID_ARGUMENT
    assert lib.bf_cuda_context_create(0, None) == _capi.BF_ERR_INVALID_ARGUMENT


def test_max_points_supports_the_benchmark_sizes():
    lib = _capi.load()
    for model in range(4):
        assert lib.bf_cuda_max_points(model) >= 4096
    assert lib.bf_cuda_max_points(9) == 0


def test_context_without_device_is_unavailable():
    lib = _capi.load()
    if lib.bf_cuda_available():
        pytest.skip("a CUDA device is present")
    ctx = C.c_void_p()
    assert lib.bf_cuda_context_create(0, C.byref(ctx)) == _capi.BF_ERR_UNAVAILABLE
    assert b"unavailable" in lib.bf_cuda_last_error()


def test_host_alloc_zero_bytes_is_a_no_op():
    lib = _capi.load()
    p = C.c_void_p(1)
    assert lib.bf_cuda_host_alloc(0, C.byref(p)) == _capi.BF_OK and not p.value
    assert lib.bf_cuda_host_free(None) == _capi.BF_OK
