"""The grading helpers in batchfit_b200/accuracy.py: the vectorised float64 model
and Jacobian against the oracle's, and the float32-equivalence criterion."""

import numpy as np
import pytest

from batchfit_b200 import accuracy as A

PARAMS = {
    "gaussian": [2.0, 0.3, 0.8],
    "lorentzian": [1.5, -0.4, 0.6],
    "pseudo_voigt": [3.0, 0.2, 1.1, 0.35],
    "two_lorentzian": [2.0, -2.0, 0.7, 1.2, 1.5, 0.5, 0.3, 0.01],
}


@pytest.mark.parametrize("model", list(PARAMS))
def test_model_and_jacobian_match_the_oracle(oracle, model):
    x = np.linspace(-5, 5, 41)
    p = np.array(PARAMS[model])
    f, J = A.model_and_jacobian(model, x, p)
    f_ref = oracle.eval_model(model, x, p, np.float64)
    J_ref = np.stack([oracle.jacobian(model, v, p, np.float64) for v in x])
    np.testing.assert_allclose(f, f_ref, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(J, J_ref, rtol=1e-11, atol=1e-13)


def test_float32_equivalence_at_the_float64_optimum(oracle):
    """At the float64 least-squares solution of a well-conditioned Lorentzian, a
    displacement of 1e-6 is below what float32 chi2 resolves and 1e-4 is not."""
    x = np.linspace(-5, 5, 129).astype(np.float32)
    f, _ = A.model_and_jacobian("lorentzian", x, np.array([2.0, 0.1, 0.7]))
    y = (f + 0.01 * np.random.default_rng(0).normal(size=x.size)).astype(np.float32)
    ref = oracle.fit("port", "lorentzian", x, y[None], None, None, None, np.float64).params[0]
    assert A.float32_equivalent("lorentzian", x, y, ref * (1 + 1e-6), ref)
    assert not A.float32_equivalent("lorentzian", x, y, ref * (1 + 1e-4), ref)
    assert not A.float32_equivalent("lorentzian", x, y, np.full(3, np.nan), ref)
    bound = A.chi2_error_bound("lorentzian", x, y, ref)
    assert 0 < bound < 1e-5 * float(np.sum((y - A.model_and_jacobian("lorentzian", x, ref)[0]) ** 2))


def test_summarize_definite_and_equivalent_fractions(oracle):
    """Fits the oracle leaves at max_iterations are left out of the definite-status
    agreement; an out-of-tolerance converged fit counts as equivalent only when its
    float64 chi2 is as low as the oracle's within the float32 error bound."""
    x = np.linspace(-5, 5, 129).astype(np.float32)
    rng = np.random.default_rng(1)
    ys, refs = [], []
    for c in (-0.5, 0.0, 0.5):
        f, _ = A.model_and_jacobian("lorentzian", x, np.array([2.0, c, 0.7]))
        y = (f + 0.01 * rng.normal(size=x.size)).astype(np.float32)
        ys.append(y)
        refs.append(oracle.fit("port", "lorentzian", x, y[None], None, None, None, np.float64).params[0])
    y, ref = np.stack(ys), np.stack(refs)
    ref_status = np.array([0, 0, 1])
    got = ref.copy()
    got[0] *= 1 + 1e-6  # within tolerance
    got[1] *= 1 + 1e-3  # out of tolerance, measurably worse
    got_status = np.array([0, 0, 0])
    chi2 = np.array([np.sum((y[i] - A.model_and_jacobian("lorentzian", x, ref[i])[0]) ** 2) for i in range(3)])
    s = A.summarize("lorentzian", x, y, got, got_status, chi2, ref, ref_status, chi2, x64=True)
    assert s["status_agreement"] == pytest.approx(2 / 3)
    assert s["status_agreement_definite"] == 1.0
    assert s["definite_fraction"] == pytest.approx(2 / 3)
    assert s["within_or_equivalent_fraction"] == 0.5


def test_float32_bounds_are_the_extremes_they_claim(oracle):
    """perturbation_bound is the largest first-order shift of the fixed point over
    every residual error of size u32 (|y| + |f|) (attained by the sign pattern of
    each row of (J^T J)^-1 J^T); resolution_bound is the largest move of one
    parameter on the ellipsoid dp^T J^T J dp = eps; a parameter at a bound gets 0."""
    x = np.linspace(-5, 5, 201).astype(np.float32)
    f, _ = A.model_and_jacobian("lorentzian", x, np.array([2.0, 0.3, 0.6]))
    y = (f + 0.01 * np.random.default_rng(2).normal(size=x.size)).astype(np.float32)
    ref = oracle.fit("port", "lorentzian", x, y[None], None, None, None, np.float64).params[0]
    fr, J = A.model_and_jacobian("lorentzian", x, ref)
    e = A.U32 * (np.abs(y.astype(np.float64)) + np.abs(fr))
    G = np.linalg.solve(J.T @ J, J.T)
    pb = A.perturbation_bound("lorentzian", x, y, ref)
    for k in range(3):
        dp = G @ (np.sign(G[k]) * e)  # the worst case for parameter k
        assert abs(dp[k]) == pytest.approx(pb[k], rel=1e-12)
        assert np.all(np.abs(G @ (np.random.default_rng(k).choice([-1.0, 1.0], x.size) * e)) <= pb * (1 + 1e-12))
    rb = A.resolution_bound("lorentzian", x, y, ref)
    eps = A.chi2_error_bound("lorentzian", x, y, ref)
    inv = np.linalg.inv(J.T @ J)
    for k in range(3):
        dp = np.sqrt(eps / inv[k, k]) * inv[:, k]  # on the ellipsoid, extreme in k
        assert dp @ (J.T @ J) @ dp == pytest.approx(eps, rel=1e-9)
        assert dp[k] == pytest.approx(rb[k], rel=1e-9)
    assert np.all(pb > 0) and np.all(rb > pb)  # sqrt(u32) against u32 scaling
    at_bound = A.perturbation_bound("lorentzian", x, y, ref, lower=np.array([0.0, ref[1], 0.0]))
    assert at_bound[1] == 0.0 and at_bound[0] > 0.0
    s = A.summarize("lorentzian", x, y[None], ref[None], np.array([0]), np.array([1.0]), ref[None], np.array([0]),
                    np.array([1.0]), x64=True, bounds=(np.full(3, -np.inf), np.full(3, np.inf)))
    assert s["first_order_below_tol_fraction"] == 1.0 and s["within_tol_where_first_order_below_tol"] == 1.0
