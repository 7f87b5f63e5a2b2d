"""The CPU oracle (oracle/, a C restatement of the reference CPU fitting path) is
pinned by (1) the golden fixtures the compiled reference produced
(tests/golden/make_golden.py), bit for bit, and (2) the known answers of the
reference's own tests."""

import glob
import hashlib
import os

import numpy as np
import pytest

from batchfit_b200 import workloads as W

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
FIELDS = ("params", "status", "iterations", "chi2", "covariance", "stderr", "uncertainty_status")
LINE, CONSTANT, EXPONENTIAL = 100, 101, 102


def load_fixture(path):
    d = dict(np.load(path))
    if "recipe" in d:
        y = getattr(W, str(d["recipe"]))().y
        assert hashlib.sha256(y.tobytes()).hexdigest() == str(d["y_sha256"]), "seeded generator drifted"
        d["y"] = y
    return d


def test_fixtures_present():
    assert len(GOLDEN) >= 4


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("dtype,tag", [(np.float32, "f32"), (np.float64, "f64")])
def test_port_matches_reference_fixture(oracle, path, dtype, tag):
    d = load_fixture(path)
    model = str(d["model"])
    r = oracle.fit("port", model, d["x"], d["y"], None, d["lower"], d["upper"], dtype, uncertainties=True)
    for field in FIELDS:
        np.testing.assert_array_equal(getattr(r, field), d[f"{tag}_{field}"], err_msg=field)
    gp, gs, gb = oracle.guess("port", model, d["x"], d["y"], dtype)
    np.testing.assert_array_equal(gp, d[f"{tag}_guess_params"])
    np.testing.assert_array_equal(gs, d[f"{tag}_guess_status"])
    np.testing.assert_array_equal(gb, d[f"{tag}_guess_baseline"])


def test_port_matches_compiled_reference_random(oracle):
    if not oracle.ref_available():
        pytest.skip("compiled reference not built here")
    for model, m in (("lorentzian", 129), ("pseudo_voigt", 512), ("gaussian", 200), ("two_lorentzian", 301)):
        rng = np.random.default_rng(m)
        x = np.linspace(-8, 8, m).astype(np.float32)
        c, w, a = rng.uniform(-3, 3, 300), rng.uniform(0.3, 2, 300), rng.uniform(0.5, 3, 300)
        y = a[:, None] / (1 + ((x[None] - c[:, None]) / w[:, None]) ** 2)
        if model == "two_lorentzian":
            y = y + 0.5 * a[:, None] / (1 + ((x[None] - c[:, None] - 3 * w[:, None]) / w[:, None]) ** 2)
        y = (y + 0.02 * rng.normal(size=y.shape)).astype(np.float32)
        for dtype in (np.float32, np.float64):
            a_ = oracle.fit("ref", model, x, y, None, None, None, dtype, uncertainties=True, workers=2)
            b_ = oracle.fit("port", model, x, y, None, None, None, dtype, uncertainties=True)
            for field in FIELDS:
                np.testing.assert_array_equal(getattr(a_, field), getattr(b_, field))


# ---- known answers from the reference's own tests --------------------------------

@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_cholesky_known_answers(oracle, dtype):
    # tests/solver_checks.hpp:44-55
    ok, _, b = oracle.cholesky_solve("port", [[4, 12, -16], [12, 37, -43], [-16, -43, 98]], [-20, -43, 192],
                                     dtype=dtype)
    assert ok
    np.testing.assert_allclose(b, [1, 2, 3], atol=1e-6)
    assert not oracle.cholesky_solve("port", [[1, 2], [2, 1]], [1, 2], dtype=dtype)[0]
    assert not oracle.cholesky_solve("port", [[1, 1], [1, 1]], [1, 2], dtype=dtype)[0]


@pytest.mark.parametrize("scaled", [False, True])
def test_scaled_cholesky_known_answer(oracle, scaled):
    # tests/numerics_checks.hpp:99-106
    ok, _, b = oracle.cholesky_solve("port", [[4, 1, 0], [1, 3, 1], [0, 1, 2]], [6, 10, 8], scaled=scaled)
    assert ok
    np.testing.assert_allclose(b, [1, 2, 3], atol=1e-14, rtol=1e-14)


def test_kahan_known_answer(oracle):
    # tests/numerics_checks.hpp:96-98: 1e8 + 1000 * 1 keeps the small terms
    assert oracle.kahan_add_f32([1.0] * 1000, start=1e8) == np.float32(100001000)


@pytest.mark.parametrize("dtype,tol", [(np.float32, 2e-6), (np.float64, 1e-14)])
def test_model_hand_values(oracle, dtype, tol):
    # tests/model_checks.hpp:54-85
    ev = lambda model, x, p: float(oracle.eval_model(model, [x], p, dtype)[0])  # noqa: E731
    single = [4, 1, 2]
    assert abs(ev("gaussian", 1, single) - 4) <= tol * 5
    assert abs(ev("gaussian", 3, single) - 4 * np.exp(-0.5)) <= tol * 5
    assert abs(ev("lorentzian", 1, single) - 4) <= tol * 5
    assert abs(ev("lorentzian", 3, single) - 2) <= tol * 5
    voigt = [4, 1, 2, 0.25]
    assert abs(ev("pseudo_voigt", 1, voigt) - 4) <= tol * 5
    assert abs(ev("pseudo_voigt", 2, voigt) - 2) <= tol * 5
    assert abs(ev("pseudo_voigt", 3, voigt) - 0.3875) <= tol * 5
    pair = [4, 1, 2, 3, -1, 1, 0.5, -0.25]
    assert abs(ev("two_lorentzian", 1, pair) - 4.85) <= tol * 5
    assert abs(ev("two_lorentzian", -1, pair) - 5.75) <= tol * 5


@pytest.mark.parametrize("model", ["gaussian", "lorentzian", "pseudo_voigt", "two_lorentzian"])
def test_jacobian_finite_differences(oracle, model):
    # tests/model_checks.hpp: analytic df/dp agrees with central differences
    rng = np.random.default_rng(4)
    p = {"gaussian": 3, "lorentzian": 3, "pseudo_voigt": 4, "two_lorentzian": 8}[model]
    for _ in range(200):
        params = np.array([rng.uniform(-5, 5), rng.uniform(-4, 4), rng.uniform(0.3, 3), rng.uniform(0, 1),
                           rng.uniform(-4, 4), rng.uniform(0.3, 3), rng.uniform(-2, 2), rng.uniform(-1, 1)])[:p]
        if model == "two_lorentzian":
            params[3] = rng.uniform(-5, 5)
        x = rng.uniform(-6, 6)
        jac = oracle.jacobian(model, x, params)
        for k in range(p):
            h = 1e-6 * max(1.0, abs(params[k]))
            up, dn = params.copy(), params.copy()
            up[k] += h
            dn[k] -= h
            fd = (oracle.eval_model(model, [x], up)[0] - oracle.eval_model(model, [x], dn)[0]) / (2 * h)
            assert abs(fd - jac[k]) <= 1e-6 + 1e-5 * abs(fd)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_guess_hand_values(oracle, dtype):
    # tests/initial_guess_checks.hpp:22-61
    tol = 2e-6 if dtype == np.float32 else 1e-12
    x = np.arange(9)
    y = [[2, 2, 2, 4, 6, 4, 2, 2, 2]]
    g, s, b = oracle.guess("port", "gaussian", x, y, dtype)
    lo, _, _ = oracle.guess("port", "lorentzian", x, y, dtype)
    pv, _, _ = oracle.guess("port", "pseudo_voigt", x, y, dtype)
    assert s[0] == 0 and abs(b[0] - 2) <= tol
    np.testing.assert_allclose(g[0], [4, 4, 2 / 2.354820045030949382], atol=tol)
    assert abs(lo[0, 2] - 1) <= tol and abs(pv[0, 2] - 2) <= tol and pv[0, 3] == 0.5
    c, s, _ = oracle.guess("port", "lorentzian", x, [[1, 1, 1, 4, 5, 3.5, 1, 1, 1]], dtype)
    assert s[0] == 0
    assert abs(c[0, 1] - 37.5 / 9.5) <= tol and abs(c[0, 2] - (5.2 - 8.0 / 3) / 2) <= tol
    n, s, _ = oracle.guess("port", "lorentzian", [10, 11, 12, 14, 15, 16, 18, 19, 20], y, dtype)
    assert s[0] == 0 and abs(n[0, 1] - 15) <= tol and abs(n[0, 2] - 1) <= tol
    flat, s, _ = oracle.guess("port", "gaussian", x, [np.zeros(9)], dtype)
    assert s[0] == 2 and np.all(np.isnan(flat))
    for bad in ([0, 1, 1, 3, 4, 5, 6, 7, 8], [0, 1, -1, 3, 4, 5, 6, 7, 8], [0, 1, np.inf, 3, 4, 5, 6, 7, 8]):
        assert oracle.guess("port", "gaussian", bad, y, dtype)[1][0] == 1
    assert oracle.guess("port", "gaussian", x[:4], [[1, 2, 1, 0]], dtype)[1][0] == 1


def test_row_statuses(oracle):
    # python/tests/test_api.py:79-87
    x = np.linspace(-4, 4, 129)
    y = np.tile(2 / (1 + ((x - 0.2) / 0.7) ** 2), (5, 1))
    y[1, 10], y[2, 10], y[3] = np.nan, np.inf, 0
    p0 = np.tile([1.8, 0, 0.8], (5, 1))
    for dtype in (np.float32, np.float64):
        r = oracle.fit("port", "lorentzian", x, y, p0, None, None, dtype)
        np.testing.assert_array_equal(r.status, [0, 3, 3, 4, 0])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stop_rules_and_bounds(oracle, dtype):
    # tests/solver_checks.hpp:175-257 on the Constant and Line models
    x, y = [-1, 0, 1], [[3, 3, 3]]
    r = oracle.fit("port", CONSTANT, x, y, [0], [0], [2], dtype)
    assert r.status[0] == 0 and r.params[0, 0] == 2 and abs(r.chi2[0] - 3) < 1e-6
    r = oracle.fit("port", CONSTANT, x, y, [99], [1], [1], dtype)
    assert r.status[0] == 0 and r.params[0, 0] == 1 and r.iterations[0] == 0 and abs(r.chi2[0] - 12) < 1e-6
    r = oracle.fit("port", CONSTANT, x, [[-3, -3, -3]], [0], [-2], [2], dtype)
    assert r.status[0] == 0 and r.params[0, 0] == -2
    aff = oracle.fit("port", LINE, [0, 1, 2], [[3, 5, 7]], [0, 0], [0, -np.inf], [2, np.inf], dtype)
    assert aff.status[0] == 0 and aff.params[0, 0] == 2
    assert abs(aff.params[0, 1] - 2.6) < 2e-5 and abs(aff.chi2[0] - 1.2) < 2e-6
    o = oracle.make_options(gradient_tolerance=10, dtype=dtype)
    r = oracle.fit("port", CONSTANT, x, y, [0], None, None, dtype, options=o)
    assert r.status[0] == 0 and r.iterations[0] == 0 and r.params[0, 0] == 0
    o = oracle.make_options(gradient_tolerance=0, cost_tolerance=0, step_tolerance=10, dtype=dtype)
    assert oracle.fit("port", CONSTANT, x, y, [0], None, None, dtype, options=o).iterations[0] == 1
    o = oracle.make_options(gradient_tolerance=0, step_tolerance=0, cost_tolerance=1, dtype=dtype)
    assert oracle.fit("port", CONSTANT, x, y, [0], None, None, dtype, options=o).iterations[0] == 1
    eps = np.finfo(dtype).eps
    o = oracle.make_options(initial_lambda=16 / eps, max_iterations=3, dtype=dtype)
    r = oracle.fit("port", CONSTANT, x, y, [0], None, None, dtype, options=o)
    assert r.status[0] == 1 and r.iterations[0] == 3


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_failure_statuses(oracle, dtype):
    # tests/solver_checks.hpp:259-346
    x, y = [1, 1, 1], [[2, 2, 2]]
    o = oracle.make_options(max_iterations=0, dtype=dtype)
    r = oracle.fit("port", CONSTANT, x, y, [0], None, None, dtype, options=o)
    assert r.status[0] == 1 and r.iterations[0] == 0 and r.chi2[0] == 12
    ey = [[np.exp(2.0)] * 3]
    o = oracle.make_options(max_iterations=1, dtype=dtype)
    r = oracle.fit("port", EXPONENTIAL, x, ey, [-2], None, None, dtype, options=o)
    assert r.status[0] == 1 and r.iterations[0] == 1 and r.params[0, 0] == -2
    o = oracle.make_options(max_iterations=200, dtype=dtype)
    r = oracle.fit("port", EXPONENTIAL, x, ey, [-2], None, None, dtype, options=o)
    assert r.status[0] == 0 and r.iterations[0] > 1 and abs(r.params[0, 0] - 2) < 1e-5
    s = oracle.fit("port", "lorentzian", [0, 0, 0], y, [1, 0, 1], None, None, dtype)
    assert s.status[0] == 2 and s.iterations[0] == 1 and s.chi2[0] == 3
    np.testing.assert_array_equal(s.params[0], [1, 0, 1])
    for lo, hi, init, opts in (([2], [1], [0], None), ([np.nan], [np.inf], [0], None), ([np.inf], [np.inf], [0], None),
                               ([-np.inf], [-np.inf], [0], None), ([-np.inf], [np.inf], [np.nan], None),
                               ([-np.inf], [np.inf], [0], oracle.make_options(initial_lambda=0, dtype=dtype))):
        r = oracle.fit("port", CONSTANT, x, y, init, lo, hi, dtype, options=opts)
        assert r.status[0] == 3 and r.iterations[0] == 0 and np.isnan(r.chi2[0])
    z = oracle.fit("port", "gaussian", [0, 0, 0], y, [1, 0, 0], None, None, dtype)
    assert z.status[0] == 3


def test_unresolved_and_degenerate(oracle):
    # python/tests/test_api.py:269-274 and tests/numerics_checks.hpp:16-62
    x = np.linspace(-1, 1, 129)
    y = 2 / (1 + (x / 1e-4) ** 2)
    r = oracle.fit("port", "lorentzian", x, [y], [2, 0, 1e-4], None, None, np.float64)
    assert r.status[0] == 5 and np.isfinite(r.chi2[0])
    for flat in (0.0, 3.0):
        r = oracle.fit("port", "lorentzian", x, [np.full(129, flat)], [2, 0, 0.2], None, None, np.float32)
        assert r.status[0] == 4


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_line_covariance_known_answer(oracle, dtype):
    # tests/uncertainty_checks.hpp:20-72: cov = SSE/(M-P) (J^T J)^-1 = 0.4 / 0.2 / 0.15
    x = [-2, -1, 0, 1, 2]
    cov, se, us = oracle.uncertainty(LINE, x, [1, 2], 0, 6, [-np.inf] * 2, [np.inf] * 2, dtype)
    assert us == 0
    assert abs(cov[0, 0] - 0.4) <= 1e-7 + 1e-6 * 0.4 and abs(cov[1, 1] - 0.2) <= 1e-7 + 1e-6 * 0.2
    assert cov[0, 1] == 0 and cov[1, 0] == 0
    cov, se, us = oracle.uncertainty(LINE, x, [1, 2], 0, 6, [1, -np.inf], [1, np.inf], dtype)
    assert us == 0 and se[0] == 0 and abs(cov[1, 1] - 0.15) <= 1e-6
    cov, se, us = oracle.uncertainty(LINE, x, [1, 2], 0, 6, [1, 2], [1, 2], dtype)
    assert us == 0 and se[1] == 0
    assert oracle.uncertainty(LINE, x[:2], [1, 2], 0, 6, [-np.inf] * 2, [np.inf] * 2, dtype)[2] == 2
    assert oracle.uncertainty(LINE, x, [1, 2], 0, 6, [1, -np.inf], [np.inf] * 2, dtype)[2] == 4
    assert oracle.uncertainty(LINE, x, [1, 2], 1, 6, [-np.inf] * 2, [np.inf] * 2, dtype)[2] == 1
    assert oracle.uncertainty(LINE, x, [1, 2], 0, np.nan, [-np.inf] * 2, [np.inf] * 2, dtype)[2] == 5
    cov, se, us = oracle.uncertainty(LINE, x, [1, 2], 0, 0, [-np.inf] * 2, [np.inf] * 2, dtype)
    assert us == 0 and se[0] == 0
