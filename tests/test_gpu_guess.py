"""The GPU data-only guess equals the reference float guess bit for bit
(initial_guess<float,Model>, include/batchfit/cpu/initial_guess.hpp:120-249),
parameters and guess status, including every failure path."""

import numpy as np
import pytest

from batchfit_b200 import workloads as W

pytestmark = pytest.mark.gpu


def check_guess(bf, oracle, model, x, y):
    got_p, got_s = bf.guess(x, y, model)
    ref_p, ref_s, _ = oracle.guess("port", model, x, y, np.float32)
    np.testing.assert_array_equal(got_s, ref_s)
    # NaN == NaN positions and bit-identical finite values.
    np.testing.assert_array_equal(got_p, ref_p)
    return got_s


def test_guess_lorentzian_small(bf, oracle):
    w = W.lorentzian_small()
    s = check_guess(bf, oracle, "lorentzian", w.x, w.y)
    assert np.all(s == 0)


def test_guess_pseudo_voigt_plain(bf, oracle):
    w = W.pseudo_voigt_plain(n=4000)
    check_guess(bf, oracle, "pseudo_voigt", w.x, w.y)


@pytest.mark.parametrize("model", ["gaussian", "lorentzian", "pseudo_voigt", "two_lorentzian"])
@pytest.mark.parametrize("m", [5, 7, 33, 64, 129, 300, 701, 1024, 1601, 2603])
def test_guess_random_shapes(bf, oracle, model, m):
    rng = np.random.default_rng(1000 + m)
    n = 257
    x = np.linspace(-10, 10, m).astype(np.float32)
    c = rng.uniform(-5, 5, n)
    w = np.exp(rng.uniform(np.log(0.2), np.log(3), n))
    a = rng.uniform(0.5, 4, n)
    y = a[:, None] / (1 + ((x[None] - c[:, None]) / w[:, None]) ** 2)
    if model == "two_lorentzian":
        c2 = c + rng.uniform(1, 4, n) * w
        y = y + 0.6 * a[:, None] / (1 + ((x[None] - c2[:, None]) / w[:, None]) ** 2)
    y = y + rng.uniform(0.0, 0.05, n)[:, None] * rng.normal(size=y.shape) + rng.uniform(-1, 1, n)[:, None] * 0.2
    y = y.astype(np.float32)
    y[3] = 0.0  # flat rows
    y[4] = 1.5
    y[5, m // 2] = np.nan  # non-finite row
    y[6, 0] = np.inf
    check_guess(bf, oracle, model, x, y)


def test_guess_two_lorentzian_cube(bf, oracle):
    w = W.two_lorentzian_cube(n=3000)
    s = check_guess(bf, oracle, "two_lorentzian", w.x, w.y)
    assert set(np.unique(s)) <= {0, 1, 2, 3}


def test_guess_hand_features(bf, oracle):
    # initial_guess_checks.hpp:22-61
    x = np.arange(9, dtype=np.float32)
    y = np.array([[2, 2, 2, 4, 6, 4, 2, 2, 2], [1, 1, 1, 4, 5, 3.5, 1, 1, 1]], np.float32)
    for model in ("gaussian", "lorentzian", "pseudo_voigt"):
        check_guess(bf, oracle, model, x, y)
    p, s = bf.guess(x, y[:1], "lorentzian")
    assert s[0] == 0 and p[0, 0] == 4 and p[0, 1] == 4 and p[0, 2] == 1
    xn = np.array([10, 11, 12, 14, 15, 16, 18, 19, 20], np.float32)
    p, s = bf.guess(xn, y[:1], "lorentzian")
    assert s[0] == 0 and abs(p[0, 1] - 15) < 2e-6 and abs(p[0, 2] - 1) < 2e-6
    # invalid grids (repeated, decreasing, infinite) and too few samples
    for bad in (np.array([0, 1, 1, 3, 4, 5, 6, 7, 8]), np.array([0, 1, -1, 3, 4, 5, 6, 7, 8]),
                np.array([0, 1, np.inf, 3, 4, 5, 6, 7, 8])):
        _, s = bf.guess(bad.astype(np.float32), y[:1], "gaussian")
        assert s[0] == 1
    _, s = bf.guess(x[:4], y[:1, :4], "gaussian")
    assert s[0] == 1


def test_guess_paired_features(bf, oracle):
    # initial_guess_checks.hpp:63-126 shapes: separated peaks, a monotonic wing,
    # a weak resolved secondary, three peaks, and a dense grid with a shoulder bump.
    def two(x, p):
        return p[0] / (1 + ((x - p[1]) / p[2]) ** 2) + p[3] / (1 + ((x - p[4]) / p[5]) ** 2) + p[6] + p[7] * x

    rows = []
    x = np.linspace(-5, 5, 201).astype(np.float32)
    for rev in (False, True):
        rows.append(two(x, [2 if rev else 3, -1.5, 0.4, 3 if rev else 2, 1.5, 0.5, 0.3, -0.04]))
    rows.append(0.2 + 2 / (1 + ((x - 0) / 0.5) ** 2))
    y = np.array(rows, np.float32)
    check_guess(bf, oracle, "two_lorentzian", x, y)
    x2 = np.linspace(-10, 10, 201).astype(np.float32)
    rows = [two(x2, [100, -2, 0.2, 1, 2, 0.2, 0, 0]),
            3 / (1 + ((x2 + 3) / 0.3) ** 2) + 2 / (1 + (x2 / 0.3) ** 2) + 1 / (1 + ((x2 - 3) / 0.3) ** 2)]
    check_guess(bf, oracle, "two_lorentzian", x2, np.array(rows, np.float32))
    xd = np.linspace(-5, 5, 2049).astype(np.float32)
    yd = two(xd, [3, -1.5, 0.7, 1, 1.5, 0.7, 0.4, 0]) + 0.3 * np.exp(-0.5 * ((xd + 2.25) / 0.015) ** 2)
    check_guess(bf, oracle, "two_lorentzian", xd, yd[None].astype(np.float32))


# Samples per group lane (1 + lane + k*G, the second-peak candidate bits) at 32 and 33,
# 96 and 97 for the 8-, 16- and 32-lane guess shapes, and the largest single-call M.
@pytest.mark.parametrize("m", [258, 259, 1538, 1539, 3074, 3075, 5129])
def test_guess_two_lorentzian_candidate_words(bf, oracle, m):
    x, y = W.noisy_doublets(m, 96, seed=m)
    s = check_guess(bf, oracle, "two_lorentzian", x, y)
    assert np.count_nonzero(s == 0) >= 40
