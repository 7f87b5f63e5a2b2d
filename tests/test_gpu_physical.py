"""Fits of float64 data in normalised coordinates (the reference's Coordinates,
include/batchfit/coordinates.hpp:15-113): the GPU normalisation and the mapping
back equal the same recipe done in numpy around an ordinary fit; on badly scaled
physical data (x offset by 1000, amplitudes of 1e4) the results match the float64
oracle run on the raw data, which a float32 fit of the raw data does not."""

import numpy as np
import pytest

from batchfit_b200 import accuracy as A

pytestmark = pytest.mark.gpu


def physical_data(n=400, m=384, seed=7):
    rng = np.random.default_rng(seed)
    x = np.linspace(1000.0, 1010.0, m)
    a = rng.uniform(5e3, 2e4, n)[:, None]
    c = rng.uniform(1002.0, 1008.0, n)[:, None]
    w = rng.uniform(0.3, 1.2, n)[:, None]
    eta = rng.uniform(0.1, 0.9, n)[:, None]
    z = (x - c) / w
    y = a * ((1 - eta) * np.exp(-4 * np.log(2) * z * z) + eta / (1 + 4 * z * z)) + 50.0 * rng.normal(size=(n, m))
    return x, y


def numpy_recipe(bf, x, y, bounds):
    """Coordinates::from / physical in numpy, around bf.fit on float32 data."""
    lo, hi = x.min(), x.max()
    half = hi / 2 - lo / 2
    origin = (lo + hi) / 2
    ys = np.abs(y).max(axis=1)
    ys = np.where(ys > 0, ys, 1.0)
    xn = ((x - origin) / half).astype(np.float32)
    yn = (y / ys[:, None]).astype(np.float32)
    r = bf.fit(xn, yn, "pseudo_voigt", None, bounds, uncertainties=True)
    q = r.params.astype(np.float64)
    params = np.column_stack([q[:, 0] * ys, q[:, 1] * half + origin, q[:, 2] * half, q[:, 3]])
    return r, params, r.chi2.astype(np.float64) * ys * ys, ys, half


def test_matches_numpy_recipe(bf):
    x, y = physical_data()
    bounds = ([0, -1, 1e-3, 0], [np.inf, 1, 2, 1])
    got = bf.fit_physical(x, y, "pseudo_voigt", None, bounds, uncertainties=True)
    r, params, chi2, ys, half = numpy_recipe(bf, x, y, bounds)
    np.testing.assert_array_equal(got.status, r.status)
    np.testing.assert_array_equal(got.iterations, r.iterations)
    np.testing.assert_allclose(got.params, params, rtol=1e-14, atol=1e-12)
    np.testing.assert_allclose(got.chi2, chi2, rtol=1e-14)
    t = np.stack([np.diag([s, half, half, 1.0]) for s in ys])
    cov = t @ r.covariance.astype(np.float64) @ t
    ok = r.uncertainty_status == 0
    np.testing.assert_allclose(got.covariance[ok], cov[ok], rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(got.stderr[ok], np.sqrt(np.einsum("nii->ni", cov[ok])), rtol=1e-12)


def test_badly_scaled_data_matches_float64_oracle(bf, oracle):
    x, y = physical_data(n=300)
    bounds = ([0, -1, 1e-3, 0], [np.inf, 1, 2, 1])
    got = bf.fit_physical(x, y, "pseudo_voigt", None, bounds)
    half = 5.0
    lo = np.array([0, -np.inf, 1e-3 * half, 0], np.float64)
    hi = np.array([np.inf, np.inf, 2 * half, 1], np.float64)
    p0, _, _ = oracle.guess("port", "pseudo_voigt", x, y, np.float64)
    ref = oracle.fit("port", "pseudo_voigt", x, y, p0, lo, hi, np.float64)
    s = A.summarize("pseudo_voigt", x, y, got.params, got.status, got.chi2, ref.params, ref.status, ref.chi2,
                    1e-4, 1e-5)
    assert s["status_agreement"] >= 0.99, s
    assert s["within_tol_fraction"] >= 0.99, s


def test_refusals(bf):
    x = np.linspace(0, 1, 16)
    with pytest.raises(ValueError, match="finite"):
        bf.fit_physical(x, np.full((2, 16), np.nan), "gaussian")
    with pytest.raises(ValueError, match="range"):
        bf.fit_physical(np.zeros(16), np.ones((2, 16)), "gaussian")
