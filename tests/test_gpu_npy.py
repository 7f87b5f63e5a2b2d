"""Out-of-core fits from .npy files: the streamed results equal, bit for bit, the
results of ``fit`` on the same arrays, for float32 and float64 inputs, ragged last
chunks, given initial values and uncertainties; existing output directories are
refused and a failed run leaves no directory behind."""

import subprocess
import sys

import numpy as np
import pytest

from batchfit_b200 import workloads as W

pytestmark = pytest.mark.gpu


def data(n, m, dtype, seed=3):
    w = W.pseudo_voigt_plain(n=n, m=m, seed=seed)
    return w, w.x.astype(dtype), w.y.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("chunk", [0, 333])
def test_streamed_equals_in_memory(bf, tmp_path, dtype, chunk):
    w, x, y = data(1000, 257, dtype)
    np.save(tmp_path / "x.npy", x)
    np.save(tmp_path / "y.npy", y)
    out = tmp_path / "out"
    s = bf.fit_npy(tmp_path / "x.npy", tmp_path / "y.npy", out, "pseudo_voigt", bounds=(w.lower, w.upper),
                   uncertainties=True, chunk_fits=chunk, in_flight=2)
    assert s["fits"] == 1000 and s["chunks"] == (1 if chunk == 0 else 4)
    ref = bf.fit(x.astype(np.float32), y.astype(np.float32), "pseudo_voigt", None, (w.lower, w.upper),
                 uncertainties=True)
    np.testing.assert_array_equal(np.load(out / "parameters.npy"), ref.params)
    np.testing.assert_array_equal(np.load(out / "chi_squared.npy"), ref.chi2)
    status = np.load(out / "status.npy")
    assert status.dtype == np.uint32 and np.load(out / "iterations.npy").dtype == np.uint32
    np.testing.assert_array_equal(status, ref.status.astype(np.uint32))
    np.testing.assert_array_equal(np.load(out / "iterations.npy"), ref.iterations)
    np.testing.assert_array_equal(np.load(out / "covariance.npy"), ref.covariance)
    np.testing.assert_array_equal(np.load(out / "standard_errors.npy"), ref.stderr)
    np.testing.assert_array_equal(np.load(out / "uncertainty_status.npy"), ref.uncertainty_status.astype(np.uint32))


def test_initial_values_and_cli(bf, tmp_path):
    w, x, y = data(500, 129, np.float32, seed=5)
    p0, _ = bf.guess(x, y, "pseudo_voigt")
    p0 = np.where(np.isfinite(p0), p0 * 1.01, p0).astype(np.float64)
    for name, arr in (("x", x), ("y", y), ("p0", p0)):
        np.save(tmp_path / f"{name}.npy", arr)
    out = tmp_path / "cli"
    res = subprocess.run([sys.executable, "-m", "batchfit_b200.npy", "--x", str(tmp_path / "x.npy"), "--y",
                          str(tmp_path / "y.npy"), "--initial", str(tmp_path / "p0.npy"), "--output", str(out),
                          "--model", "pseudo_voigt", "--chunk-fits", "128"], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert res.stdout.startswith("fits=500 chunks=4 chunk_fits=128")
    ref = bf.fit(x, y, "pseudo_voigt", p0.astype(np.float32))
    np.testing.assert_array_equal(np.load(out / "parameters.npy"), ref.params)
    np.testing.assert_array_equal(np.load(out / "status.npy"), ref.status.astype(np.uint32))


def test_refusals(bf, tmp_path):
    w, x, y = data(10, 64, np.float32)
    np.save(tmp_path / "x.npy", x)
    np.save(tmp_path / "y.npy", y)
    (tmp_path / "exists").mkdir()
    with pytest.raises(ValueError, match="must not already exist"):
        bf.fit_npy(tmp_path / "x.npy", tmp_path / "y.npy", tmp_path / "exists", "gaussian")
    np.save(tmp_path / "x2.npy", x[:-1])
    with pytest.raises(ValueError, match="shape"):
        bf.fit_npy(tmp_path / "x2.npy", tmp_path / "y.npy", tmp_path / "out2", "gaussian")
    assert not (tmp_path / "out2").exists()
    np.save(tmp_path / "p0.npy", np.zeros((10, 2), np.float32))
    with pytest.raises(ValueError, match="initial"):
        bf.fit_npy(tmp_path / "x.npy", tmp_path / "y.npy", tmp_path / "out3", "gaussian", initial=tmp_path / "p0.npy")
    assert not (tmp_path / "out3").exists()
