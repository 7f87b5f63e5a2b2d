"""The native .npy header reader (host only, no GPU): numpy's own files are read
as the reference's npy::inspect reads them (src/cpu/npy.cpp:50-91), and
unsupported files are refused with a message."""

import ctypes as C

import numpy as np
import pytest

from batchfit_b200 import _capi


def inspect(path):
    lib = _capi.load()
    dtype, rank, shape = C.c_int32(), C.c_int32(), (C.c_uint64 * 2)()
    rc = lib.bf_npy_inspect(str(path).encode(), C.byref(dtype), C.byref(rank), shape)
    if rc != 0:
        raise ValueError(_capi.last_error())
    return dtype.value, rank.value, (shape[0], shape[1])


@pytest.mark.parametrize("dtype,code", [(np.float32, 0), (np.float64, 1), (np.uint32, 2)])
@pytest.mark.parametrize("shape", [(7,), (5, 3), (0, 4), (1, 1)])
def test_numpy_files(tmp_path, dtype, code, shape):
    p = tmp_path / "a.npy"
    np.save(p, np.zeros(shape, dtype))
    d, r, s = inspect(p)
    assert d == code and r == len(shape)
    assert s == (shape[0], shape[1] if len(shape) == 2 else 0)


def test_format_2_header(tmp_path):
    p = tmp_path / "v2.npy"
    with open(p, "wb") as f:
        np.lib.format.write_array(f, np.ones((3, 2), np.float32), version=(2, 0))
    assert inspect(p) == (0, 2, (3, 2))


@pytest.mark.parametrize("make,match", [
    (lambda p: np.save(p, np.zeros((2, 3), np.int64)), "dtype"),
    (lambda p: np.save(p, np.asfortranarray(np.zeros((2, 3), np.float32))), "fortran"),
    (lambda p: np.save(p, np.zeros((2, 3, 4), np.float32)), "shape"),
    (lambda p: np.save(p, np.zeros((2, 3), ">f4")), "dtype"),
    (lambda p: open(p, "wb").write(b"not an npy file"), "NPY"),
])
def test_refused(tmp_path, make, match):
    p = tmp_path / "bad.npy"
    make(p)
    with pytest.raises(ValueError, match=match):
        inspect(p)


def test_truncated_payload(tmp_path):
    p = tmp_path / "t.npy"
    np.save(p, np.zeros((4, 4), np.float32))
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-4])
    with pytest.raises(ValueError, match="payload"):
        inspect(p)
