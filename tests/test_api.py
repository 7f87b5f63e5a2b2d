"""Host-side contract of batchfit_b200.fit (mirrors python/tests/test_api.py of the
reference): argument errors raise before any device work, explicit CUDA never
falls back, and the result types match the reference's."""

import numpy as np
import pytest

import batchfit_b200 as bf


def data(n=8):
    x = np.linspace(-4, 4, 129)
    y = np.tile(2 / (1 + ((x - 0.2) / 0.7) ** 2), (n, 1))
    return x, y


@pytest.mark.parametrize("change,error", [
    ({"model": "missing"}, ValueError), ({"device": "gpu"}, ValueError), ({"device": "cpu"}, ValueError),
    ({"device": "metal"}, ValueError), ({"p0": [1, 2]}, ValueError), ({"bounds": ([0, 0], [1, 1])}, ValueError),
    ({"bounds": (3, 2)}, ValueError), ({"bounds": (np.nan, np.inf)}, ValueError),
    ({"bounds": (-np.inf, 1e300)}, ValueError), ({"policy": "fast"}, ValueError),
])
def test_invalid_options(change, error):
    x, y = data()
    with pytest.raises(error):
        bf.fit(x, y, **{"device": "cuda", **change})


@pytest.mark.parametrize("x,y,error", [
    (np.zeros((2, 2)), np.zeros((2, 2)), ValueError), ([], [], ValueError), ([1, 2], [[1, 2, 3]], ValueError),
    ([1j, 2j], [[1, 2]], TypeError), ([1, 2], [["a", "b"]], TypeError),
])
def test_invalid_arrays(x, y, error):
    with pytest.raises(error):
        bf.fit(x, y, device="cuda")


def test_uncertainty_flag_is_explicit_boolean():
    with pytest.raises(TypeError, match="boolean"):
        bf.fit([0, 1, 2], [1, 2, 1], uncertainties="yes")


def test_explicit_cuda_never_falls_back():
    x, y = data()
    if bf.cuda_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match="unavailable"):
        bf.fit(x, y, p0=[1.8, 0, 0.8], device="cuda")


def test_result_types_and_enums():
    assert bf.FitResult._fields == ("params", "status", "iterations", "chi2")
    assert bf.FitResultWithUncertainties._fields[4:] == ("covariance", "stderr", "uncertainty_status")
    assert [s.value for s in bf.FitStatus] == list(range(6))
    assert bf.FitStatus.unresolved_peak == 5 and bf.UncertaintyStatus.active_bound == 4
    assert bf.MODELS == {"gaussian": 0, "lorentzian": 1, "pseudo_voigt": 2, "two_lorentzian": 3}


def test_solver_options_overrides():
    o = bf.solver_options("pseudo_voigt", [0, -1, 0, 0], [1, 1, 1, 1], "reference", max_iterations=7)
    assert o.max_iterations == 7 and o.policy == 0 and list(o.lower)[:4] == [0, -1, 0, 0]
    with pytest.raises(ValueError):
        bf.solver_options("pseudo_voigt", [0] * 4, [1] * 4, "reference", bogus=1)
