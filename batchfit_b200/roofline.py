"""Algorithmic work of the bounded-LM fit path, for roofline fractions.

Work is counted from the reference's formulas (include/batchfit/models.hpp:78-185)
and the reference solver's pass structure (include/batchfit/cpu/solver.hpp:145-192):

* a *cost* pass evaluates the model and accumulates r^2 (detail::cost);
* a *linearize* pass evaluates model + analytic Jacobian and accumulates J^T r and
  the lower triangle of J^T J (detail::linearize);
* the covariance re-linearises once more (Jacobian + J^T J only,
  include/batchfit/cpu/uncertainty.hpp:42-52).

Per fit: M * (L * linearize + C * cost + U * jacobian) where L and C are the pass
counts of the float64 oracle's own trajectory on the same data (so the GPU's own
iteration count can neither inflate nor deflate its roofline) and U = 1 with
uncertainties.  Flops count each add, multiply and division as one and a written
a*b+c as two; exp() and the model's non-constant reciprocal are MUFU operations,
counted separately.  The GPU kernel's compensation, reductions and FP64 control
are not algorithmic work.
"""

from __future__ import annotations

from dataclasses import dataclass

# Per-point (flops, mufu) of the reference formulas; the Jacobian reuses the
# shared subexpressions (z, exp, reciprocal) of the value in the same pass.
#                  eval            jacobian extra   accumulate g, A (lower)
_COUNTS = {
    # z=(x-c)/s: 2; -0.5*z*z: 2; exp; *A: 1  | A*G*z/s: 3, *z: 1          | P=3: g 6, A 12
    "gaussian": {"eval": (5, 1), "jac": (4, 0), "p": 3},
    # z: 2; 1+z*z: 2; A/(...): rcp 1 + mul 1 | 2*A*S*S/s: 4, *z: 1, *z: 1 | P=3
    "lorentzian": {"eval": (5, 1), "jac": (6, 0), "p": 3},
    # z: 2; -4ln2*z*z: 2; 1+4*z*z: 3; (1-e)g+el, *A: 5; exp, rcp | scale 7, *z 1, *z 1, A*(l-g) 2 | P=4
    "pseudo_voigt": {"eval": (12, 2), "jac": (11, 0), "p": 4},
    # two Lorentzians (2x 5) + intercept + slope*x (3) | 2x6 Jacobian extras | P=8
    "two_lorentzian": {"eval": (13, 2), "jac": (12, 0), "p": 8},
}


@dataclass(frozen=True)
class PointWork:
    linearize_flops: int
    cost_flops: int
    jacobian_flops: int
    mufu_per_eval: int


def point_work(model: str) -> PointWork:
    c = _COUNTS[model]
    p = c["p"]
    eval_f, mufu = c["eval"]
    jac_f, _ = c["jac"]
    acc_g = 2 * p
    acc_a = 2 * p * (p + 1) // 2
    residual = 1
    return PointWork(
        linearize_flops=eval_f + jac_f + residual + acc_g + acc_a,
        cost_flops=eval_f + residual + 2,
        jacobian_flops=eval_f + jac_f + acc_a,
        mufu_per_eval=mufu,
    )


def fit_work(model: str, m: int, linearize_passes: float, cost_passes: float, uncertainties: bool):
    """(flops, mufu_ops) of one fit with M points, given the oracle's mean pass counts."""
    w = point_work(model)
    u = 1 if uncertainties else 0
    flops = m * (linearize_passes * w.linearize_flops + cost_passes * w.cost_flops + u * w.jacobian_flops)
    mufu = m * w.mufu_per_eval * (linearize_passes + cost_passes + u)
    return flops, mufu


def observation_bytes(m: int, p: int, uncertainties: bool) -> int:
    """HBM bytes of one fit: y read once, outputs written (p0 absent: guesses)."""
    out = 4 * p + 12
    if uncertainties:
        out += 4 * (p * p + p + 1)
    return 4 * m + out
