"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (numpy PCG64; no dataset is involved).

* ``lorentzian_small``      Lorentzian, N=1000, M=129 on linspace(-5,5); y = 2/(1+((x-c)/0.7)^2)
                             with c = linspace(-0.5,0.5,N) + 0.02*N(0,1) (seed 123).
* ``pseudo_voigt_plain``    pseudo-Voigt, M=512 on linspace(-10,10); A~U[0.5,5], c~U[-6,6],
                             FWHM~logU[0.1,3], mixing~U[0,1], noise sigma = 1% of A (seed 2).
* ``two_lorentzian_cube``   two Lorentzians (P=8, intercept=slope=0 in the data), M=1024 on
                             linspace(-20,20); HWHM~logU[0.2,2], separation U[0.5,3]*HWHM, amplitude
                             ratio U[0.1,1]; 5% pure-noise rows and 2% constant rows; noise sigma
                             0.5% of the largest amplitude (seed 3).
* ``mixed_stream``          mixed models (25% each), per-fit M~logU[64,4096] on its own
                             linspace(-10,10,M) (seed 4).

Every generator returns float32 arrays; the float64 oracle promotes the same values.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BOUNDS = {
    "lorentzian_small": ([0.0, -5.0, 1e-4], [np.inf, 5.0, 5.0]),
    "pseudo_voigt_plain": ([0.0, -10.0, 1e-3, 0.0], [np.inf, 10.0, 10.0, 1.0]),
    "two_lorentzian_cube": ([0.0, -20.0, 1e-3, 0.0, -20.0, 1e-3, -np.inf, -np.inf],
                            [np.inf, 20.0, 20.0, np.inf, 20.0, 20.0, np.inf, np.inf]),
}


@dataclass
class Workload:
    name: str
    model: str
    x: np.ndarray
    y: np.ndarray
    lower: np.ndarray
    upper: np.ndarray
    truth: np.ndarray | None = None
    meta: dict = field(default_factory=dict)


def _bounds(name):
    lo, hi = BOUNDS[name]
    return np.asarray(lo, np.float32), np.asarray(hi, np.float32)


def lorentzian_small(n=1000, seed=123):
    x = np.linspace(-5, 5, 129)
    c = np.linspace(-0.5, 0.5, n)
    clean = 2.0 / (1.0 + ((x[None, :] - c[:, None]) / 0.7) ** 2)
    rng = np.random.default_rng(seed)
    y = clean + 0.02 * rng.normal(size=clean.shape)
    lo, hi = _bounds("lorentzian_small")
    truth = np.column_stack([np.full(n, 2.0), c, np.full(n, 0.7)])
    return Workload("lorentzian_small", "lorentzian", x.astype(np.float32), y.astype(np.float32), lo, hi,
                    truth.astype(np.float32))


def _pv(x, a, c, w, eta):
    z = (x[None, :] - c[:, None]) / w[:, None]
    g = np.exp(-4.0 * np.log(2.0) * z * z)
    l = 1.0 / (1.0 + 4.0 * z * z)
    return a[:, None] * ((1.0 - eta[:, None]) * g + eta[:, None] * l)


def pseudo_voigt_plain(n=1_000_000, m=512, seed=2, chunk=65536):
    """The 1M-fit pseudo-Voigt throughput workload (generated in row chunks)."""
    rng = np.random.default_rng(seed)
    x64 = np.linspace(-10, 10, m)
    a = rng.uniform(0.5, 5.0, n)
    c = rng.uniform(-6.0, 6.0, n)
    w = np.exp(rng.uniform(np.log(0.1), np.log(3.0), n))
    eta = rng.uniform(0.0, 1.0, n)
    y = np.empty((n, m), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        clean = _pv(x64, a[s:e], c[s:e], w[s:e], eta[s:e])
        y[s:e] = clean + (0.01 * a[s:e])[:, None] * rng.normal(size=clean.shape)
    lo, hi = _bounds("pseudo_voigt_plain")
    truth = np.column_stack([a, c, w, eta]).astype(np.float32)
    return Workload("pseudo_voigt_plain", "pseudo_voigt", x64.astype(np.float32), y, lo, hi, truth)


def _lor(x, a, c, w):
    z = (x[None, :] - c[:, None]) / w[:, None]
    return a[:, None] / (1.0 + z * z)


def two_lorentzian_cube(n=262_144, m=1024, seed=3, chunk=32768):
    rng = np.random.default_rng(seed)
    x64 = np.linspace(-20, 20, m)
    w1 = np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))
    w2 = np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))
    sep = rng.uniform(0.5, 3.0, n) * 0.5 * (w1 + w2)
    c1 = rng.uniform(-12.0, 12.0, n)
    c2 = c1 + sep
    a1 = rng.uniform(0.5, 5.0, n)
    a2 = a1 * rng.uniform(0.1, 1.0, n)
    kind = rng.uniform(size=n)
    noise_only = kind < 0.05
    constant = (kind >= 0.05) & (kind < 0.07)
    level = rng.uniform(0.0, 1.0, n)
    y = np.empty((n, m), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        clean = _lor(x64, a1[s:e], c1[s:e], w1[s:e]) + _lor(x64, a2[s:e], c2[s:e], w2[s:e])
        sigma = 0.005 * np.maximum(a1[s:e], a2[s:e])
        noisy = clean + sigma[:, None] * rng.normal(size=clean.shape)
        pure = sigma[:, None] * rng.normal(size=clean.shape)
        block = np.where(noise_only[s:e, None], pure, noisy)
        block = np.where(constant[s:e, None], level[s:e, None], block)
        y[s:e] = block
    lo, hi = _bounds("two_lorentzian_cube")
    truth = np.column_stack([a1, c1, w1, a2, c2, w2, np.zeros(n), np.zeros(n)]).astype(np.float32)
    return Workload("two_lorentzian_cube", "two_lorentzian", x64.astype(np.float32), y, lo, hi, truth,
                    {"noise_only": noise_only, "constant": constant})


def noisy_doublets(m, n, seed):
    """Two-Lorentzian rows, from resolved to merged, with noise strong enough that
    most candidates of the second-peak search are noise maxima."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-10, 10, m).astype(np.float32)
    c = rng.uniform(-5, 5, n)[:, None]
    w = np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))[:, None]
    a = rng.uniform(0.5, 4, n)[:, None]
    c2 = c + rng.uniform(0.3, 4.0, n)[:, None] * w
    y = a / (1 + ((x - c) / w) ** 2) + rng.uniform(0.1, 1.0, n)[:, None] * a / (1 + ((x - c2) / w) ** 2)
    y = y + rng.uniform(0.005, 0.2, n)[:, None] * a * rng.normal(size=y.shape)
    return x, y.astype(np.float32)


MODEL_NAMES = ("gaussian", "lorentzian", "pseudo_voigt", "two_lorentzian")
MIXED_BOUNDS = {
    "gaussian": ([0.0, -10.0, 1e-3], [np.inf, 10.0, 10.0]),
    "lorentzian": ([0.0, -10.0, 1e-3], [np.inf, 10.0, 10.0]),
    "pseudo_voigt": ([0.0, -10.0, 1e-3, 0.0], [np.inf, 10.0, 10.0, 1.0]),
    "two_lorentzian": ([0.0, -10.0, 1e-3, 0.0, -10.0, 1e-3, -np.inf, -np.inf],
                       [np.inf, 10.0, 10.0, np.inf, 10.0, 10.0, np.inf, np.inf]),
}


@dataclass
class MixedWorkload:
    """Uneven batch: fit i has model models[i] and M = counts[i] points at
    x[offsets[i]:offsets[i]+counts[i]] and y[offsets[i]:...] (one concatenated buffer)."""

    models: np.ndarray
    counts: np.ndarray
    offsets: np.ndarray
    x: np.ndarray
    y: np.ndarray


def mixed_stream(n=65_536, seed=4, m_min=64, m_max=4096):
    rng = np.random.default_rng(seed)
    models = rng.integers(0, 4, n).astype(np.int32)
    counts = np.exp(rng.uniform(np.log(m_min), np.log(m_max), n)).astype(np.int64)
    counts = np.clip(counts, m_min, m_max)
    offsets = np.zeros(n, np.int64)
    offsets[1:] = np.cumsum(counts)[:-1]
    total = int(counts.sum())
    x = np.empty(total, np.float32)
    y = np.empty(total, np.float32)
    for i in range(n):
        m = int(counts[i])
        xi = np.linspace(-10, 10, m)
        a = rng.uniform(0.5, 5.0)
        c = rng.uniform(-6.0, 6.0)
        w = np.exp(rng.uniform(np.log(0.1), np.log(3.0)))
        kind = models[i]
        if kind == 0:
            clean = a * np.exp(-0.5 * ((xi - c) / (w / 2.354820045)) ** 2)
        elif kind == 1:
            clean = a / (1 + ((xi - c) / (w / 2)) ** 2)
        elif kind == 2:
            z = (xi - c) / w
            eta = rng.uniform()
            clean = a * ((1 - eta) * np.exp(-4 * np.log(2) * z * z) + eta / (1 + 4 * z * z))
        else:
            w2 = np.exp(rng.uniform(np.log(0.2), np.log(2.0)))
            c2 = c + rng.uniform(0.5, 3.0) * 0.5 * (w / 2 + w2)
            a2 = a * rng.uniform(0.1, 1.0)
            clean = a / (1 + ((xi - c) / (w / 2)) ** 2) + a2 / (1 + ((xi - c2) / w2) ** 2)
        s = offsets[i]
        x[s:s + m] = xi
        y[s:s + m] = clean + 0.01 * a * rng.normal(size=m)
    return MixedWorkload(models, counts.astype(np.int32), offsets, x, y)


# ----------------------------------------------------------------- serving --
SERVING_M = (64, 105, 172, 283, 463, 760, 1248, 2048)  # log-spaced over [64, 2048]


def _mixed_rows(model, x, n, rng):
    """n spectra of `model` on x with the mixed stream's parameter distributions."""
    a = rng.uniform(0.5, 5.0, n)[:, None]
    c = rng.uniform(-6.0, 6.0, n)[:, None]
    w = np.exp(rng.uniform(np.log(0.1), np.log(3.0), n))[:, None]
    if model == "gaussian":
        clean = a * np.exp(-0.5 * ((x - c) / (w / 2.354820045)) ** 2)
    elif model == "lorentzian":
        clean = a / (1 + ((x - c) / (w / 2)) ** 2)
    elif model == "pseudo_voigt":
        z = (x - c) / w
        eta = rng.uniform(0.0, 1.0, n)[:, None]
        clean = a * ((1 - eta) * np.exp(-4 * np.log(2) * z * z) + eta / (1 + 4 * z * z))
    else:
        w2 = np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))[:, None]
        c2 = c + rng.uniform(0.5, 3.0, n)[:, None] * 0.5 * (w / 2 + w2)
        a2 = a * rng.uniform(0.1, 1.0, n)[:, None]
        clean = a / (1 + ((x - c) / (w / 2)) ** 2) + a2 / (1 + ((x - c2) / w2) ** 2)
    return (clean + 0.01 * a * rng.normal(size=clean.shape)).astype(np.float32)


@dataclass
class ServingPool:
    """Spectra for the serving stream: for every (model, M in SERVING_M) a block of
    `rows` seeded spectra, tiled to `n_max` rows so that any request is a view."""

    x: dict
    y: dict
    n_max: int


def serving_pool(rows=2048, n_max=50_000, seed=5, alloc=None):
    """``alloc(shape)`` may return pinned host arrays (default: numpy)."""
    rng = np.random.default_rng(seed)
    xs, ys = {}, {}
    for model in MODEL_NAMES:
        for m in SERVING_M:
            x = np.linspace(-10, 10, m)
            block = _mixed_rows(model, x, rows, rng)
            out = alloc((n_max, m)) if alloc else np.empty((n_max, m), np.float32)
            reps = -(-n_max // rows)
            for r in range(reps):
                lo = r * rows
                hi = min(n_max, lo + rows)
                out[lo:hi] = block[: hi - lo]
            xs[(model, m)] = x.astype(np.float32)
            ys[(model, m)] = out
    return ServingPool(xs, ys, n_max)


@dataclass
class ServingRequest:
    arrival: float  # seconds from the stream's start
    model: str
    m: int
    n: int
    uncertainties: bool


def serving_stream(rate, duration, seed=5, n_max=50_000):
    """Poisson arrivals at `rate` requests/s for `duration` s; per request N ~
    logU[1, n_max], M ~ logU[64, 2048] (snapped to SERVING_M), a random model, half
    with uncertainties."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        m_cont = np.exp(rng.uniform(np.log(64), np.log(2048)))
        m = min(SERVING_M, key=lambda v: abs(np.log(v) - np.log(m_cont)))
        n = int(np.exp(rng.uniform(0.0, np.log(n_max))))
        out.append(ServingRequest(t, MODEL_NAMES[int(rng.integers(4))], m, max(1, n), bool(rng.integers(2))))
    return out
