"""Error definitions used to grade a float32 fit against the float64 oracle.

* Parameters: relative error |d| / max(|ref|, floor_k).  Amplitudes and widths use
  floor 0 (plain relative), centers use the x span, mixing uses 1, and the
  two-Lorentzian baseline terms use the row's signal scale (intercept) and signal
  scale / x span (slope), because their reference values are ~0 by construction.
* chi2: plain relative |d| / |ref|.
* Status agreement: equal codes.

A fit "passes" when the statuses agree and, for converged reference fits, every
parameter is within ``param_tol`` and chi2 within ``chi2_tol``.
"""

from __future__ import annotations

import numpy as np

# Parameter roles per model (python/batchfit/__init__.py:13; models.hpp parameter_name).
ROLES = {
    "gaussian": ("amp", "center", "width"),
    "lorentzian": ("amp", "center", "width"),
    "pseudo_voigt": ("amp", "center", "width", "mixing"),
    "two_lorentzian": ("amp", "center", "width", "amp", "center", "width", "intercept", "slope"),
}


def floors(model, x, y=None):
    """Per-(fit, parameter) floors for the relative-error denominator."""
    span = float(np.max(x) - np.min(x))
    roles = ROLES[model]
    n = 1 if y is None else y.shape[0]
    scale = np.ones(n) if y is None else np.max(np.abs(y.astype(np.float64)), axis=1)
    out = np.zeros((n, len(roles)))
    for k, role in enumerate(roles):
        if role == "center":
            out[:, k] = span
        elif role == "mixing":
            out[:, k] = 1.0
        elif role == "intercept":
            out[:, k] = scale
        elif role == "slope":
            out[:, k] = scale / span
    return out


def param_errors(model, x, y, got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    den = np.maximum(np.abs(ref), floors(model, x, y))
    with np.errstate(divide="ignore", invalid="ignore"):
        err = np.abs(got - ref) / den
    err[(got == ref)] = 0.0
    return err


def chi2_errors(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        err = np.abs(got - ref) / np.abs(ref)
    err[got == ref] = 0.0
    return err


def summarize(model, x, y, got_params, got_status, got_chi2, ref_params, ref_status, ref_chi2,
              param_tol=1e-4, chi2_tol=1e-5):
    """Accuracy summary of a float32 result against the float64 oracle."""
    agree = np.asarray(got_status) == np.asarray(ref_status)
    converged = agree & np.isin(np.asarray(ref_status), (0, 5))
    pe = param_errors(model, x, y, got_params, ref_params)
    ce = chi2_errors(got_chi2, ref_chi2)
    pmax = np.where(converged, np.nanmax(np.where(np.isfinite(pe), pe, np.inf), axis=1), 0.0)
    cerr = np.where(converged, np.where(np.isfinite(ce), ce, np.inf), 0.0)
    within = agree & (pmax <= param_tol) & (cerr <= chi2_tol)
    n = len(agree)
    conv = max(1, int(converged.sum()))
    return {
        "n": n,
        "status_agreement": float(agree.mean()) if n else 1.0,
        "within_tol_fraction": float(within.mean()) if n else 1.0,
        "params_within_fraction": float((pmax[converged] <= param_tol).sum() / conv),
        "chi2_within_fraction": float((cerr[converged] <= chi2_tol).sum() / conv),
        "param_err_max": float(pmax[converged].max()) if converged.any() else 0.0,
        "param_err_p999": float(np.quantile(pmax[converged], 0.999)) if converged.any() else 0.0,
        "chi2_err_max": float(cerr[converged].max()) if converged.any() else 0.0,
        "param_tol": param_tol,
        "chi2_tol": chi2_tol,
    }
