"""Error definitions used to grade a float32 fit against the float64 oracle.

* Parameters: relative error |d| / max(|ref|, floor_k).  Amplitudes and widths use
  floor 0 (plain relative), centers use the x span, mixing uses 1, and the
  two-Lorentzian baseline terms use the row's signal scale (intercept) and signal
  scale / x span (slope), because their reference values are ~0 by construction.
* chi2: plain relative |d| / |ref|.
* Status agreement: equal codes.

A fit "passes" when the statuses agree and, for converged reference fits, every
parameter is within ``param_tol`` and chi2 within ``chi2_tol``.

Two further measures separate what float32 arithmetic can decide from what it
cannot (``summarize(..., x64=True)``):

* status agreement on fits with a definite float64 status: a float64 fit that
  ends at max_iterations has no status a float32 solver could be held to;
* float32 equivalence: a converged fit whose parameters miss the tolerance but
  whose float64 chi2 is no higher than the oracle's by more than the float32
  evaluation error of chi2 at the oracle's solution (``chi2_error_bound``).  Along
  the flat valleys of weakly determined fits (overlapping doublets, a component
  fitted to a noise spike) chi2 changes by less than float32 can evaluate while
  parameters move by more than 1e-4; no float32 evaluation of the model can order
  such points, so they are equally good answers to the float32 data.
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
              param_tol=1e-4, chi2_tol=1e-5, x64=False, bounds=None):
    """Accuracy summary of a float32 result against the float64 oracle.  x64 adds
    the definite-status agreement and the float32-equivalence fraction; with
    `bounds` (lower, upper) it also gives, over the oracle-converged fits, the
    two float32 bounds relative to the parameter errors' denominators: the
    first-order fixed-point bound (``perturbation_bound``), with the fraction
    within tolerance among the fits where it is below param_tol, and the chi2
    resolution (``resolution_bound``), with the same split."""
    agree = np.asarray(got_status) == np.asarray(ref_status)
    converged = agree & np.isin(np.asarray(ref_status), (0, 5))
    pe = param_errors(model, x, y, got_params, ref_params)
    ce = chi2_errors(got_chi2, ref_chi2)
    pmax = np.where(converged, np.nanmax(np.where(np.isfinite(pe), pe, np.inf), axis=1), 0.0)
    cerr = np.where(converged, np.where(np.isfinite(ce), ce, np.inf), 0.0)
    within = agree & (pmax <= param_tol) & (cerr <= chi2_tol)
    n = len(agree)
    conv = max(1, int(converged.sum()))
    extra = {}
    if x64:
        definite = np.asarray(ref_status) != 1
        equivalent = within.copy()
        for i in np.where(converged & ~within)[0]:
            equivalent[i] = float32_equivalent(model, x, y[i], got_params[i], ref_params[i])
        extra = {"status_agreement_definite": float(agree[definite].mean()) if definite.any() else 1.0,
                 "definite_fraction": float(definite.mean()) if n else 1.0,
                 "within_or_equivalent_fraction": float(equivalent[converged].sum() / conv)}
        if bounds is not None:
            ref_conv = np.isin(np.asarray(ref_status), (0, 5))
            den = floors(model, x, y)
            refp = np.asarray(ref_params, np.float64)
            rel = {"first_order": np.full(n, np.inf), "chi2_resolution": np.full(n, np.inf)}
            for i in np.where(ref_conv)[0]:
                yi = np.asarray(y[i], np.float64)
                d = np.maximum(np.abs(refp[i]), den[i])
                for name, fn in (("first_order", perturbation_bound), ("chi2_resolution", resolution_bound)):
                    b = fn(model, x, yi, refp[i], bounds[0], bounds[1])
                    with np.errstate(divide="ignore", invalid="ignore"):
                        rel[name][i] = float(np.max(np.where(b == 0.0, 0.0, b / d)))
            for name, r in rel.items():
                small = ref_conv & (r <= param_tol)
                extra[f"{name}_median"] = float(np.median(r[ref_conv])) if ref_conv.any() else 0.0
                extra[f"{name}_below_tol_fraction"] = float(small[ref_conv].mean()) if ref_conv.any() else 1.0
                extra[f"within_tol_where_{name}_below_tol"] = float(within[small].mean()) if small.any() else None
    return {**extra,
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


# ------------------------------------------------- float32 resolution of chi2 --
U32 = 2.0 ** -24  # unit roundoff of float32


def model_and_jacobian(model, x, p):
    """f(x) and df/dp (float64, vectorised over x) of the reference's model
    formulas (include/batchfit/models.hpp:78-185)."""
    x = np.asarray(x, np.float64)
    p = np.asarray(p, np.float64)
    if model in ("lorentzian", "two_lorentzian"):
        peaks = ((0, 1, 2), (3, 4, 5)) if model == "two_lorentzian" else ((0, 1, 2),)
        f = np.zeros_like(x)
        J = np.zeros((x.size, p.size))
        for ia, ic, iw in peaks:
            z = (x - p[ic]) / p[iw]
            s = 1.0 / (1.0 + z * z)
            t = 2.0 * p[ia] * s * s * z / p[iw]
            f += p[ia] * s
            J[:, ia], J[:, ic], J[:, iw] = s, t, t * z
        if model == "two_lorentzian":
            f += p[6] + p[7] * x
            J[:, 6], J[:, 7] = 1.0, x
        return f, J
    if model == "gaussian":
        z = (x - p[1]) / p[2]
        g = np.exp(-0.5 * z * z)
        t = p[0] * g * z / p[2]
        return p[0] * g, np.column_stack([g, t, t * z])
    z = (x - p[1]) / p[2]
    g = np.exp(-4.0 * np.log(2.0) * z * z)
    lo = 1.0 / (1.0 + 4.0 * z * z)
    s = (1.0 - p[3]) * g + p[3] * lo
    t = 8.0 * p[0] / p[2] * z * ((1.0 - p[3]) * np.log(2.0) * g + p[3] * lo * lo)
    return p[0] * s, np.column_stack([s, t, t * z, p[0] * (lo - g)])


def chi2_error_bound(model, x, y, params):
    """First-order bound of the error of chi2 evaluated in float32 at `params`:
    each residual y - f carries an error of at most u32 (|y| + |f|), so chi2 does
    2 u32 sum_j |r_j| (|y_j| + |f_j|)."""
    f, _ = model_and_jacobian(model, x, params)
    y = np.asarray(y, np.float64)
    return 2.0 * U32 * float(np.sum(np.abs(y - f) * (np.abs(y) + np.abs(f))))


def _free(p, lower, upper):
    free = np.ones(p.size, bool)
    if lower is not None:
        free &= p > np.asarray(lower, np.float64)
    if upper is not None:
        free &= p < np.asarray(upper, np.float64)
    return free


def perturbation_bound(model, x, y, params, lower=None, upper=None):
    """First-order bound of how far float32 evaluation moves the fixed point of a
    gradient-based solver from a float64 minimiser `params`: each residual carries
    an error of at most u32 (|y| + |f|), the stationarity condition J^T r = 0
    shifts by J^T of it, and the parameters by (J^T J)^-1 J^T of it:
    |dp_k| <= sum_i |[(J^T J)^-1 J^T]_ki| u32 (|y_i| + |f_i|), over the free
    parameters (0 at a bound, inf when J^T J is singular)."""
    p = np.asarray(params, np.float64)
    if not np.all(np.isfinite(p)):
        return np.full(p.size, np.inf)
    f, J = model_and_jacobian(model, x, p)
    free = _free(p, lower, upper)
    out = np.zeros(p.size)
    if not free.any():
        return out
    Jf = J[:, free]
    try:
        G = np.linalg.solve(Jf.T @ Jf, Jf.T)
    except np.linalg.LinAlgError:
        out[free] = np.inf
        return out
    out[free] = np.abs(G) @ (U32 * (np.abs(np.asarray(y, np.float64)) + np.abs(f)))
    return out


def resolution_bound(model, x, y, params, lower=None, upper=None):
    """Per-parameter float32 resolution at a float64 minimiser `params`: the
    largest move of parameter k that keeps the Gauss-Newton chi2 within the float32
    evaluation error of chi2 (``chi2_error_bound``), max |dp_k| subject to
    dp^T (J^T J) dp <= eps, which is sqrt(eps * [(J^T J)^-1]_kk) over the free
    parameters (strictly inside their bounds).  Parameters at a bound get 0; a
    singular J^T J gives inf.  A fit whose bound is below the tolerance is one a
    float32 solver can pin down to it; above it, float32 cannot order the points
    that separate the answers."""
    p = np.asarray(params, np.float64)
    if not np.all(np.isfinite(p)):
        return np.full(p.size, np.inf)
    _, J = model_and_jacobian(model, x, p)
    eps = chi2_error_bound(model, x, y, p)
    free = _free(p, lower, upper)
    out = np.zeros(p.size)
    if not free.any():
        return out
    Jf = J[:, free]
    try:
        inv = np.linalg.inv(Jf.T @ Jf)
    except np.linalg.LinAlgError:
        out[free] = np.inf
        return out
    d = np.diag(inv)
    out[free] = np.where(d > 0, np.sqrt(eps * np.maximum(d, 0.0)), np.inf)
    return out


def float32_equivalent(model, x, y, got, ref):
    """Whether `got` is as good a minimiser as `ref` to float32 arithmetic: its
    float64 chi2 exceeds ref's by no more than the float32 evaluation error of
    chi2 at ref."""
    y = np.asarray(y, np.float64)
    got = np.asarray(got, np.float64)
    if not np.all(np.isfinite(got)):
        return False
    c_ref = float(np.sum((y - model_and_jacobian(model, x, ref)[0]) ** 2))
    c_got = float(np.sum((y - model_and_jacobian(model, x, got)[0]) ** 2))
    return c_got <= c_ref + chi2_error_bound(model, x, y, ref)
