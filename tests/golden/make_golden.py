"""Regenerate the golden fixtures in this directory from the reference itself.

    make -C oracle REFERENCE=<batchfit tree>   # builds oracle/_ref/libbatchfit_ref.so from the reference sources
    python tests/golden/make_golden.py

Each fixture holds seeded float32 inputs and the reference's own outputs
(cpu::fit_batch<float> and <double> after initial_guess, with uncertainties, and
initial_guess<float>/<double> alone), computed by the compiled reference C++ via
oracle/_ref.  The CPU test suite checks the oracle's C restatement against them
bit for bit, so the restatement stays pinned where the reference tree is absent.
"""

from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from batchfit_b200 import workloads as W  # noqa: E402
from oracle import pyoracle as O  # noqa: E402


def cases():
    w = W.lorentzian_small()
    yield "lorentzian_small", w.model, w.x, w.y, w.lower, w.upper
    w = W.pseudo_voigt_plain(n=48, seed=2)
    yield "pseudo_voigt_plain_48", w.model, w.x, w.y, w.lower, w.upper
    w = W.two_lorentzian_cube(n=48, seed=3)
    yield "two_lorentzian_cube_48", w.model, w.x, w.y, w.lower, w.upper
    rng = np.random.default_rng(20261109)
    x = np.linspace(-5, 5, 129).astype(np.float32)
    c, s, a = rng.uniform(-1, 1, 64), rng.uniform(0.4, 1.2, 64), rng.uniform(1, 3, 64)
    y = a[:, None] * np.exp(-0.5 * ((x[None] - c[:, None]) / s[:, None]) ** 2)
    y = (y + 0.03 * rng.normal(size=y.shape)).astype(np.float32)
    y[5] = 0.0
    y[6, 40] = np.nan
    yield "gaussian_129", "gaussian", x, y, np.array([0, -5, 0.01], np.float32), np.array([np.inf, 5, 5], np.float32)


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle REFERENCE=<batchfit tree>")
    for name, model, x, y, lo, hi in cases():
        out = {"model": np.array(model), "x": x, "lower": lo, "upper": hi}
        if name == "lorentzian_small":
            # Large and fully determined by its seed: store a digest, regenerate in tests.
            out["recipe"] = np.array(name)
            out["y_sha256"] = np.array(hashlib.sha256(y.tobytes()).hexdigest())
        else:
            out["y"] = y
        for dtype, tag in ((np.float32, "f32"), (np.float64, "f64")):
            r = O.fit("ref", model, x, y, None, lo, hi, dtype, uncertainties=True, workers=2)
            for field in ("params", "status", "iterations", "chi2", "covariance", "stderr", "uncertainty_status"):
                out[f"{tag}_{field}"] = getattr(r, field)
            gp, gs, gb = O.guess("ref", model, x, y, dtype)
            out[f"{tag}_guess_params"], out[f"{tag}_guess_status"], out[f"{tag}_guess_baseline"] = gp, gs, gb
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
