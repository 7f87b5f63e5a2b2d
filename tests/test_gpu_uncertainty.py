"""Monte-Carlo coverage of the GPU's standard errors: the reference gates every
device's covariance on it (python/tests/test_uncertainty.py:101-118).  10,000
noisy realisations of one spectrum per model; the truth must lie within one
standard error of the fitted value for 68.27% +- 2 percentage points of them, per
parameter, with no failed fit or unavailable uncertainty discarded."""

import numpy as np
import pytest

from batchfit_b200 import accuracy as A

pytestmark = pytest.mark.gpu

MODELS = ("gaussian", "lorentzian", "pseudo_voigt", "two_lorentzian")
# Truth and initial values of the reference's coverage test
# (python/tests/test_uncertainty.py:12-23).
TRUTH = {
    "gaussian": [2, .2, .7],
    "lorentzian": [2, .2, .7],
    "pseudo_voigt": [2, .2, 1.4, .5],
    "two_lorentzian": [2, -1.5, .5, 1.7, 1.5, .6, .25, .01],
}
INITIAL = {
    "gaussian": [1.8, 0, .8],
    "lorentzian": [1.8, 0, .8],
    "pseudo_voigt": [1.8, 0, 1.6, .45],
    "two_lorentzian": [1.8, -1.3, .55, 1.5, 1.3, .7, .2, 0],
}


def domain(model):
    """Bounds of the reference's test (python/tests/test_uncertainty.py:26-35)."""
    p = len(TRUTH[model])
    lower, upper = np.full(p, -np.inf, np.float32), np.full(p, np.inf, np.float32)
    lower[0], lower[2] = 0, 1e-4
    lower[1], upper[1] = -5, 5
    if p == 4:
        lower[3], upper[3] = 0, 1
    if p == 8:
        lower[3], lower[5], lower[4], upper[4] = 0, 1e-4, -5, 5
    return lower, upper


@pytest.mark.parametrize("model", MODELS)
def test_monte_carlo_10000_coverage(bf, model):
    n = 10_000
    rng = np.random.default_rng(20261110 + MODELS.index(model))
    truth = np.asarray(TRUTH[model], np.float64)
    x = np.linspace(-5, 5, 129)
    clean, _ = A.model_and_jacobian(model, x, truth)
    y = (clean + rng.normal(0, .03, (n, x.size))).astype(np.float32)
    r = bf.fit(x.astype(np.float32), y, model, np.asarray(INITIAL[model], np.float32), domain(model), "cuda",
               uncertainties=True)
    available = (r.status == bf.FitStatus.converged) & (r.uncertainty_status == bf.UncertaintyStatus.available)
    inside = available[:, None] & np.isfinite(r.stderr) & (np.abs(r.params - truth) <= r.stderr)
    coverage = np.count_nonzero(inside, axis=0) / n  # failed or unavailable rows are misses
    assert np.all(available), "no failed fit or unavailable uncertainty may be discarded"
    assert np.all(np.abs(coverage - 0.682689492137) <= .02), coverage
