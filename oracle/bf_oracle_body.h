/* Type-generic body of the oracle, included by bf_oracle.c once with REAL=float and
 * once with REAL=double.  Test infrastructure only (see bf_oracle.h).
 *
 * Every arithmetic expression keeps the reference's association order and uses no
 * FMA contraction (Makefile: -ffp-contract=off), so that each result rounds exactly
 * as the reference's C++ does on x86-64.
 *
 * Required macros: REAL, F(name) (suffixes a name), REAL_EPS, REAL_MAX, REAL_MIN,
 * EXPR(x) (expf/exp), SQRTR(x), FABSR(x), ISFINR(x), NANR.
 */

/* ---------------------------------------------------------------- models --- */
/* include/batchfit/models.hpp:78-100 (Gaussian), :102-125 (Lorentzian),
 * :127-157 (PseudoVoigt), :159-185 (TwoLorentzian).  LN2 is the host macro at :11. */
#define BFO_LN2 0.693147180559945309417232121458176568

static REAL F(lor_eval)(REAL x, const REAL *p) {
    const REAL z = (x - p[1]) / p[2];
    return p[0] / ((REAL)1 + z * z);
}

static void F(lor_jac)(REAL x, const REAL *p, REAL *out) {
    const REAL z = (x - p[1]) / p[2];
    const REAL shape = (REAL)1 / ((REAL)1 + z * z);
    const REAL scale = (REAL)2 * p[0] * shape * shape / p[2];
    out[0] = shape;
    out[1] = scale * z;
    out[2] = scale * z * z;
}

REAL F(bfo_eval)(int model, REAL x, const REAL *p) {
    switch (model) {
    case BFO_LINE: /* uncertainty_checks.hpp:8-15, solver_checks.hpp:32-39 */
        return p[0] + p[1] * x;
    case BFO_CONSTANT: /* solver_checks.hpp:22-26 */
        return p[0];
    case BFO_EXPONENTIAL: /* solver_checks.hpp:27-31 */
        return EXPR(x * p[0]);
    case 0: {
        const REAL z = (x - p[1]) / p[2];
        return p[0] * EXPR(-(REAL)0.5f * z * z);
    }
    case 1:
        return F(lor_eval)(x, p);
    case 2: {
        const REAL z = (x - p[1]) / p[2];
        const REAL g = EXPR(-(REAL)4 * (REAL)BFO_LN2 * z * z);
        const REAL l = (REAL)1 / ((REAL)1 + (REAL)4 * z * z);
        return p[0] * (((REAL)1 - p[3]) * g + p[3] * l);
    }
    default:
        return F(lor_eval)(x, p) + F(lor_eval)(x, p + 3) + p[6] + p[7] * x;
    }
}

void F(bfo_jacobian)(int model, REAL x, const REAL *p, REAL *out) {
    switch (model) {
    case BFO_LINE:
        out[0] = (REAL)1;
        out[1] = x;
        return;
    case BFO_CONSTANT:
        out[0] = (REAL)1;
        return;
    case BFO_EXPONENTIAL:
        out[0] = x * EXPR(x * p[0]);
        return;
    case 0: {
        const REAL z = (x - p[1]) / p[2];
        const REAL shape = EXPR(-(REAL)0.5f * z * z);
        out[0] = shape;
        out[1] = p[0] * shape * z / p[2];
        out[2] = p[0] * shape * z * z / p[2];
        return;
    }
    case 1:
        F(lor_jac)(x, p, out);
        return;
    case 2: {
        const REAL z = (x - p[1]) / p[2];
        const REAL g = EXPR(-(REAL)4 * (REAL)BFO_LN2 * z * z);
        const REAL l = (REAL)1 / ((REAL)1 + (REAL)4 * z * z);
        const REAL scale = p[0] * (REAL)8 / p[2] *
                           (((REAL)1 - p[3]) * (REAL)BFO_LN2 * g + p[3] * l * l);
        out[0] = ((REAL)1 - p[3]) * g + p[3] * l;
        out[1] = scale * z;
        out[2] = scale * z * z;
        out[3] = p[0] * (l - g);
        return;
    }
    default:
        F(lor_jac)(x, p, out);
        F(lor_jac)(x, p + 3, out + 3);
        out[6] = (REAL)1;
        out[7] = x;
        return;
    }
}

/* ------------------------------------------------------------- numerics --- */
/* numerics::add, include/batchfit/numerics.hpp:12-18 (Kahan). */
static void F(kahan)(REAL term, REAL *sum, REAL *correction) {
    const REAL adjusted = term - *correction;
    const REAL next = *sum + adjusted;
    *correction = (next - *sum) - adjusted;
    *sum = next;
}

/* std::clamp(v, lo, hi) as used by solver.hpp:228,297. */
static REAL F(clampr)(REAL v, REAL lo, REAL hi) { return v < lo ? lo : (hi < v ? hi : v); }
/* std::max / std::min argument semantics (first argument wins ties / NaN compares). */
static REAL F(maxr)(REAL a, REAL b) { return a < b ? b : a; }
static REAL F(minr)(REAL a, REAL b) { return b < a ? b : a; }

/* ------------------------------------------------------------- solver.hpp --- */
/* grid_spacing, solver.hpp:58-69. */
static REAL F(grid_spacing)(const REAL *x, size_t m) {
    REAL spacing = (REAL)INFINITY;
    int up = 1, down = 1;
    for (size_t j = 1; j < m; ++j) {
        const REAL d = x[j] - x[j - 1];
        up = up && d >= (REAL)0;
        down = down && d <= (REAL)0;
        if (d != (REAL)0)
            spacing = F(minr)(spacing, FABSR(d));
    }
    return (up || down) && ISFINR(spacing) ? spacing : (REAL)0;
}

/* free_shape, solver.hpp:70-82. */
static int F(free_shape)(int model, const REAL *lo, const REAL *hi) {
    int free = lo[1] != hi[1] || lo[2] != hi[2];
    if (model == 2)
        free = free || lo[3] != hi[3];
    if (model == 3)
        free = free || lo[4] != hi[4] || lo[5] != hi[5];
    return free;
}

/* spectral_success, solver.hpp:83-96: 5 = unresolved_peak, 0 = converged. */
static int32_t F(spectral_success)(int model, const REAL *p, REAL spacing) {
    if (!bfo_spectral(model))
        return 0;
    const REAL factor = model == 0   ? (REAL)2.354820045030949382
                        : model == 2 ? (REAL)1
                                     : (REAL)2;
    if (spacing > (REAL)0 && FABSR(p[2]) * factor < spacing)
        return 5;
    if (model == 3 && spacing > (REAL)0 && FABSR(p[5]) * factor < spacing)
        return 5;
    return 0;
}

/* cholesky_solve, solver.hpp:98-143; a is row-major PxP (lower triangle becomes L). */
static int F(cholesky)(unsigned p, REAL *a, REAL *rhs, int scaled) {
    REAL scale[8];
    if (scaled) {
        for (unsigned i = 0; i < p; ++i) {
            if (!ISFINR(a[i * p + i]) || a[i * p + i] <= (REAL)0)
                return 0;
            scale[i] = SQRTR(a[i * p + i]);
        }
        for (unsigned i = 0; i < p; ++i) {
            rhs[i] /= scale[i];
            for (unsigned j = 0; j < p; ++j)
                a[i * p + j] = (a[i * p + j] / scale[i]) / scale[j];
        }
    }
    for (unsigned i = 0; i < p; ++i) {
        for (unsigned j = 0; j <= i; ++j) {
            REAL value = a[i * p + j];
            for (unsigned k = 0; k < j; ++k)
                value -= a[i * p + k] * a[j * p + k];
            if (!ISFINR(value) || (i == j && value <= (REAL)0))
                return 0;
            a[i * p + j] = i == j ? SQRTR(value) : value / a[j * p + j];
        }
        REAL value = rhs[i];
        for (unsigned j = 0; j < i; ++j)
            value -= a[i * p + j] * rhs[j];
        rhs[i] = value / a[i * p + i];
    }
    for (unsigned i = p; i-- > 0;) {
        REAL value = rhs[i];
        for (unsigned j = i + 1; j < p; ++j)
            value -= a[j * p + i] * rhs[j];
        rhs[i] = value / a[i * p + i];
        if (!ISFINR(rhs[i]))
            return 0;
    }
    if (scaled)
        for (unsigned i = 0; i < p; ++i) {
            rhs[i] /= scale[i];
            if (!ISFINR(rhs[i]))
                return 0;
        }
    return 1;
}

int F(bfo_cholesky_solve)(unsigned p, REAL *matrix, REAL *rhs, int scaled) {
    if (p == 0 || p > 8)
        return -1;
    return F(cholesky)(p, matrix, rhs, scaled);
}

/* detail::cost, solver.hpp:145-157. */
static REAL F(cost)(int model, const REAL *x, const REAL *y, size_t m, const REAL *p,
                    int compensated) {
    REAL value = 0, correction = 0;
    for (size_t j = 0; j < m; ++j) {
        const REAL r = y[j] - F(bfo_eval)(model, x[j], p);
        if (compensated)
            F(kahan)(r * r, &value, &correction);
        else
            value += r * r;
    }
    return value;
}

/* detail::linearize, solver.hpp:159-192: a (PxP, mirrored), g = J^T r. */
static int F(linearize)(int model, unsigned p, const REAL *x, const REAL *y, size_t m,
                        const REAL *params, REAL *a, REAL *g, int compensated) {
    REAL ac[64], gc[8];
    for (unsigned k = 0; k < p * p; ++k)
        a[k] = ac[k] = 0;
    for (unsigned k = 0; k < p; ++k)
        g[k] = gc[k] = 0;
    for (size_t j = 0; j < m; ++j) {
        const REAL r = y[j] - F(bfo_eval)(model, x[j], params);
        REAL jac[8];
        F(bfo_jacobian)(model, x[j], params, jac);
        for (unsigned k = 0; k < p; ++k) {
            if (compensated)
                F(kahan)(jac[k] * r, &g[k], &gc[k]);
            else
                g[k] += jac[k] * r;
            for (unsigned l = 0; l <= k; ++l) {
                if (compensated)
                    F(kahan)(jac[k] * jac[l], &a[k * p + l], &ac[k * p + l]);
                else
                    a[k * p + l] += jac[k] * jac[l];
            }
        }
    }
    for (unsigned k = 0; k < p; ++k) {
        if (!ISFINR(g[k]))
            return 0;
        for (unsigned l = 0; l <= k; ++l) {
            if (!ISFINR(a[k * p + l]))
                return 0;
            a[l * p + k] = a[k * p + l];
        }
    }
    return 1;
}

typedef struct F(opts) {
    unsigned max_iterations;
    REAL lambda0, gtol, xtol, ftol;
    int compensated, scaled;
    REAL lo[8], hi[8];
} F(opts);

/* fit_single, solver.hpp:195-342.  Returns status; fills p, iterations, chi2. */
static int32_t F(fit_single)(int model, unsigned p, const REAL *x, const REAL *y, size_t m,
                             const REAL *initial, const F(opts) * o, REAL *params,
                             uint32_t *iterations, REAL *chi2, bfo_counters *counters) {
    *iterations = 0;
    *chi2 = NANR;
    for (unsigned k = 0; k < p; ++k)
        params[k] = initial[k];
    if (m == 0 || !ISFINR(o->lambda0) || o->lambda0 <= (REAL)0)
        return 3;
    const REAL tols[3] = {o->gtol, o->xtol, o->ftol};
    for (int t = 0; t < 3; ++t)
        if (!ISFINR(tols[t]) || tols[t] < (REAL)0)
            return 3;
    for (unsigned k = 0; k < p; ++k)
        if (!ISFINR(initial[k]) || isnan(o->lo[k]) || isnan(o->hi[k]) || o->lo[k] > o->hi[k] ||
            o->lo[k] == (REAL)INFINITY || o->hi[k] == -(REAL)INFINITY)
            return 3;
    for (size_t j = 0; j < m; ++j)
        if (!ISFINR(x[j]) || !ISFINR(y[j]))
            return 3;
    for (unsigned k = 0; k < p; ++k)
        params[k] = F(clampr)(initial[k], o->lo[k], o->hi[k]);
    *chi2 = F(cost)(model, x, y, m, params, o->compensated);
    if (counters)
        counters->cost_passes++;
    if (!ISFINR(*chi2)) {
        *chi2 = NANR;
        return 3;
    }
    const REAL spacing = F(grid_spacing)(x, m);
    if (bfo_spectral(model)) {
        int varied = 0, flat = 1;
        for (size_t j = 0; j < m; ++j) {
            varied = varied || x[j] != x[0];
            flat = flat && y[j] == y[0];
        }
        if (varied && flat && F(free_shape)(model, o->lo, o->hi))
            return 4;
    }
    REAL lambda = o->lambda0;
    const REAL lambda_max = F(maxr)(o->lambda0, (REAL)1 / REAL_EPS);
    for (unsigned it = 0; it < o->max_iterations; ++it) {
        REAL a[64], g[8];
        if (counters)
            counters->linearize_passes++;
        if (!F(linearize)(model, p, x, y, m, params, a, g, o->compensated))
            return 3;
        int active[8];
        REAL gnorm = 0;
        for (unsigned k = 0; k < p; ++k) {
            active[k] = o->lo[k] == o->hi[k] || (params[k] == o->lo[k] && g[k] < (REAL)0) ||
                        (params[k] == o->hi[k] && g[k] > (REAL)0);
            if (!active[k])
                gnorm = F(maxr)(gnorm, FABSR(g[k]));
        }
        if (gnorm <= o->gtol)
            return F(spectral_success)(model, params, spacing);
        REAL damped[64], delta[8];
        for (unsigned k = 0; k < p * p; ++k)
            damped[k] = a[k];
        for (unsigned k = 0; k < p; ++k)
            delta[k] = g[k];
        for (unsigned k = 0; k < p; ++k) {
            if (active[k]) {
                for (unsigned l = 0; l < p; ++l)
                    damped[k * p + l] = damped[l * p + k] = (REAL)0;
                damped[k * p + k] = (REAL)1;
                delta[k] = (REAL)0;
            } else {
                damped[k * p + k] += lambda * a[k * p + k];
            }
        }
        *iterations = it + 1;
        if (!F(cholesky)(p, damped, delta, o->scaled))
            return 2;
        REAL trial[8];
        REAL step_norm = 0, param_norm = 0, predicted = 0;
        int finite_trial = 1;
        for (unsigned k = 0; k < p; ++k) {
            step_norm = F(maxr)(step_norm, FABSR(delta[k]));
            trial[k] = F(clampr)(params[k] + delta[k], o->lo[k], o->hi[k]);
            finite_trial = finite_trial && ISFINR(trial[k]);
            delta[k] = trial[k] - params[k];
            param_norm = F(maxr)(param_norm, FABSR(params[k]));
        }
        if (step_norm <= o->xtol * (param_norm + o->xtol) / F(maxr)((REAL)1, lambda))
            return F(spectral_success)(model, params, spacing);
        for (unsigned k = 0; k < p; ++k) {
            predicted += (REAL)2 * g[k] * delta[k];
            for (unsigned l = 0; l < p; ++l)
                predicted -= delta[k] * a[k * p + l] * delta[l];
        }
        REAL trial_cost = NANR;
        if (finite_trial) {
            trial_cost = F(cost)(model, x, y, m, trial, o->compensated);
            if (counters)
                counters->cost_passes++;
        }
        const REAL reduction = *chi2 - trial_cost;
        const REAL threshold = o->ftol * *chi2;
        const int small = ISFINR(trial_cost) && ISFINR(predicted) && predicted >= (REAL)0 &&
                          FABSR(reduction) <= threshold &&
                          predicted <= threshold / F(maxr)((REAL)1, lambda);
        if (ISFINR(trial_cost) && reduction > (REAL)0 && ISFINR(predicted) &&
            predicted > (REAL)0) {
            for (unsigned k = 0; k < p; ++k)
                params[k] = trial[k];
            *chi2 = trial_cost;
            const REAL ratio = reduction / predicted;
            const REAL third = (REAL)1 / (REAL)3;
            const REAL factor =
                ratio >= (REAL)1
                    ? third
                    : F(maxr)(third, (REAL)1 - ((REAL)2 * ratio - (REAL)1) *
                                                   ((REAL)2 * ratio - (REAL)1) *
                                                   ((REAL)2 * ratio - (REAL)1));
            lambda = F(clampr)(lambda * factor, REAL_EPS, lambda_max);
        } else {
            lambda = F(minr)(lambda_max, lambda * (REAL)10);
        }
        if (small)
            return F(spectral_success)(model, params, spacing);
    }
    return 1;
}

/* estimate_uncertainty, include/batchfit/cpu/uncertainty.hpp:12-110. */
static int32_t F(uncertainty)(int model, unsigned p, const REAL *x, size_t m,
                              const REAL *params, int32_t fit_status, REAL chi2, const REAL *lo,
                              const REAL *hi, REAL *cov_out, REAL *se_out) {
    for (unsigned k = 0; k < p * p; ++k)
        cov_out[k] = NANR;
    for (unsigned k = 0; k < p; ++k)
        se_out[k] = NANR;
    if (fit_status != 0)
        return 1; /* not_converged */
    if (!ISFINR(chi2) || chi2 < (REAL)0)
        return 5;
    int fixed[8];
    unsigned nfree = 0;
    for (unsigned k = 0; k < p; ++k) {
        if (!ISFINR(params[k]) || isnan(lo[k]) || isnan(hi[k]) || lo[k] > hi[k] ||
            params[k] < lo[k] || params[k] > hi[k])
            return 5;
        fixed[k] = lo[k] == hi[k];
        nfree += !fixed[k];
        if (!fixed[k] && (params[k] == lo[k] || params[k] == hi[k]))
            return 4; /* active_bound */
    }
    if (m <= nfree)
        return 2; /* insufficient_dof */
    REAL info[64], corr[64];
    for (unsigned k = 0; k < p * p; ++k)
        info[k] = corr[k] = 0;
    for (size_t j = 0; j < m; ++j) {
        if (!ISFINR(x[j]))
            return 5;
        REAL jac[8];
        F(bfo_jacobian)(model, x[j], params, jac);
        for (unsigned i = 0; i < p; ++i) {
            if (!ISFINR(jac[i]))
                return 5;
            for (unsigned l = 0; l <= i; ++l)
                F(kahan)(jac[i] * jac[l], &info[i * p + l], &corr[i * p + l]);
        }
    }
    for (unsigned i = 0; i < p; ++i)
        for (unsigned l = 0; l <= i; ++l) {
            if (!ISFINR(info[i * p + l]))
                return 5;
            info[l * p + i] = info[i * p + l];
        }
    for (unsigned i = 0; i < p; ++i)
        if (fixed[i]) {
            for (unsigned l = 0; l < p; ++l)
                info[i * p + l] = info[l * p + i] = (REAL)0;
            info[i * p + i] = (REAL)1;
        }
    const REAL variance = chi2 / (REAL)(m - nfree);
    if (!ISFINR(variance))
        return 5;
    REAL cov[64];
    for (unsigned k = 0; k < p * p; ++k)
        cov[k] = 0;
    for (unsigned column = 0; column < p; ++column) {
        if (fixed[column])
            continue;
        REAL factor[64], rhs[8];
        for (unsigned k = 0; k < p * p; ++k)
            factor[k] = info[k];
        for (unsigned k = 0; k < p; ++k)
            rhs[k] = (REAL)0;
        rhs[column] = (REAL)1;
        if (!F(cholesky)(p, factor, rhs, 1))
            return 3; /* singular_matrix */
        for (unsigned i = 0; i < p; ++i) {
            if (!fixed[i] && factor[i * p + i] * factor[i * p + i] <= (REAL)64 * REAL_EPS)
                return 3;
            cov[i * p + column] = fixed[i] ? (REAL)0 : rhs[i] * variance;
            if (!ISFINR(cov[i * p + column]))
                return 5;
        }
    }
    for (unsigned i = 0; i < p; ++i) {
        if (cov[i * p + i] < (REAL)0)
            return 5;
        for (unsigned l = 0; l < i; ++l) {
            const REAL sym = cov[i * p + l] / (REAL)2 + cov[l * p + i] / (REAL)2;
            cov[i * p + l] = cov[l * p + i] = sym;
        }
    }
    for (unsigned k = 0; k < p * p; ++k)
        cov_out[k] = cov[k];
    for (unsigned i = 0; i < p; ++i)
        se_out[i] = SQRTR(cov[i * p + i]);
    return 0; /* available */
}

int F(bfo_uncertainty)(int model, size_t m, const REAL *x, const REAL *params,
                       int32_t fit_status, REAL chi2, const REAL *lower, const REAL *upper,
                       REAL *covariance, REAL *stderr_out, int32_t *ustatus) {
    if (!bfo_known(model))
        return 1;
    *ustatus = F(uncertainty)(model, bfo_pcount(model), x, m, params, fit_status, chi2, lower,
                              upper, covariance, stderr_out);
    return 0;
}

/* ------------------------------------------------------- initial_guess.hpp --- */
/* std::midpoint for floating point (C++20 [numeric.ops.midpoint]): the correctly
 * rounded (a+b)/2 away from overflow/underflow. */
static REAL F(midpoint)(REAL a, REAL b) {
    const REAL lo = REAL_MIN * (REAL)2, hi = REAL_MAX / (REAL)2;
    const REAL aa = a < 0 ? -a : a, ab = b < 0 ? -b : b;
    if (aa <= hi && ab <= hi)
        return (a + b) / (REAL)2;
    if (aa < lo)
        return a + b / (REAL)2;
    if (ab < lo)
        return a / (REAL)2 + b;
    return a / (REAL)2 + b / (REAL)2;
}

/* std::lerp (C++20 [c.math.lerp]) as libstdc++ evaluates it: the two-term form when
 * a and b straddle zero, exact at t == 1, otherwise a + t(b-a) kept monotonic
 * against b. */
static REAL F(lerp)(REAL a, REAL b, REAL t) {
    if ((a <= (REAL)0 && b >= (REAL)0) || (a >= (REAL)0 && b <= (REAL)0))
        return t * b + ((REAL)1 - t) * a;
    if (t == (REAL)1)
        return b;
    const REAL v = a + t * (b - a);
    if ((t > (REAL)1) == (b > a))
        return b < v ? v : b;
    return b > v ? v : b;
}

static int F(cmp)(const void *pa, const void *pb) {
    const REAL a = *(const REAL *)pa, b = *(const REAL *)pb;
    return (a > b) - (a < b);
}

/* detail::median, initial_guess.hpp:25-30: the order statistic (nth_element) and,
 * for even counts, the midpoint of the two central order statistics.  Sorts in place. */
static REAL F(median)(REAL *v, size_t n) {
    qsort(v, n, sizeof(REAL), F(cmp));
    const size_t mid = n / 2;
    return n % 2 ? v[mid] : F(midpoint)(v[mid - 1], v[mid]);
}

/* detail::smooth, initial_guess.hpp:32-36. */
static REAL F(smooth)(const REAL *s, size_t m, size_t i) {
    if (i == 0 || i + 1 == m)
        return s[i];
    return (REAL)0.25 * s[i - 1] + (REAL)0.5 * s[i] + (REAL)0.25 * s[i + 1];
}

/* detail::prominence, initial_guess.hpp:38-54. */
static REAL F(prominence)(const REAL *s, size_t m, size_t index) {
    const REAL height = F(smooth)(s, m, index);
    REAL left = height, right = height;
    for (size_t j = index; j > 0;) {
        const REAL value = F(smooth)(s, m, --j);
        if (value > height)
            break;
        left = F(minr)(left, value);
    }
    for (size_t j = index + 1; j < m; ++j) {
        const REAL value = F(smooth)(s, m, j);
        if (value > height)
            break;
        right = F(minr)(right, value);
    }
    return height - F(maxr)(left, right);
}

typedef struct F(peak_t) {
    REAL amplitude, center, width, left_radius, right_radius;
    int valid;
} F(peak_t);

static REAL F(crossing)(const REAL *x, const REAL *s, size_t a, size_t b, REAL half) {
    const REAL den = s[b] - s[a];
    if (!ISFINR(den) || den == (REAL)0)
        return NANR;
    return F(lerp)(x[a], x[b], (half - s[a]) / den);
}

/* detail::peak, initial_guess.hpp:61-109. */
static F(peak_t) F(peak)(const REAL *x, const REAL *s, size_t m, size_t index, size_t begin,
                         size_t end, int mirror) {
    F(peak_t) r = {0, 0, 0, 0, 0, 0};
    r.amplitude = s[index];
    if (!(r.amplitude > (REAL)0))
        return r;
    const REAL half = r.amplitude / (REAL)2;
    size_t left = index, right = index;
    while (left > begin && s[left] > half)
        --left;
    while (right < end && s[right] > half)
        ++right;
    const int has_left = s[left] <= half, has_right = s[right] <= half;
    if ((!has_left && (!mirror || begin == 0)) || (!has_right && (!mirror || end + 1 == m)) ||
        (!has_left && !has_right))
        return r;
    size_t low = index > 2 ? index - 2 : 0;
    size_t high = index + 2 < end ? index + 2 : end;
    const size_t low_limit = has_left ? left + 1 : begin;
    const size_t high_limit = has_right ? right - 1 : end;
    low = low < low_limit ? low_limit : low;
    high = high_limit < high ? high_limit : high;
    REAL total = 0;
    r.center = x[index];
    for (size_t j = low; j <= high; ++j) {
        const REAL weight = F(maxr)((REAL)0, s[j]) / r.amplitude;
        if (weight > (REAL)0) {
            total += weight;
            r.center = F(lerp)(r.center, x[j], weight / total);
        }
    }
    if (has_left)
        r.left_radius = r.center - F(crossing)(x, s, left, left + 1, half);
    if (has_right)
        r.right_radius = F(crossing)(x, s, right - 1, right, half) - r.center;
    if (!has_left)
        r.left_radius = r.right_radius;
    if (!has_right)
        r.right_radius = r.left_radius;
    r.width = r.left_radius + r.right_radius;
    r.valid = ISFINR(r.center) && ISFINR(r.width) && r.left_radius > (REAL)0 &&
              r.right_radius > (REAL)0;
    return r;
}

/* detail::raw_maximum, initial_guess.hpp:111-115: first maximum of s[i-1..i+1]. */
static size_t F(raw_maximum)(const REAL *s, size_t index) {
    size_t best = index - 1;
    for (size_t j = index; j <= index + 1; ++j)
        if (s[best] < s[j])
            best = j;
    return best;
}

/* initial_guess, initial_guess.hpp:120-249.  Returns the GuessStatus
 * (0 success, 1 invalid_input, 2 no_peak, 3 insufficient_peaks).  edges holds
 * 2*max(1,m/10) scratch values, signal m. */
static int32_t F(guess_one)(int model, const REAL *x, const REAL *y, size_t m, REAL *params,
                            REAL *baseline, REAL *edges, REAL *signal) {
    const unsigned p = bfo_pcount(model);
    const int paired = model == 3;
    for (unsigned k = 0; k < p; ++k)
        params[k] = NANR;
    *baseline = NANR;
    if (m < 5)
        return 1;
    REAL spacing = REAL_MAX;
    for (size_t j = 0; j < m; ++j) {
        if (!ISFINR(x[j]) || !ISFINR(y[j]) || (j > 0 && x[j] <= x[j - 1]))
            return 1;
        if (j > 0)
            spacing = F(minr)(spacing, x[j] - x[j - 1]);
    }
    if (!ISFINR(x[m - 1] - x[0]))
        return 1;
    const size_t count = m / 10 > 1 ? m / 10 : 1;
    for (size_t j = 0; j < count; ++j) {
        edges[j] = y[j];
        edges[count + j] = y[m - count + j];
    }
    const REAL left_level = F(median)(edges, count);
    const REAL right_level = F(median)(edges + count, count);
    *baseline = F(median)(edges, 2 * count);
    const REAL left_x = F(midpoint)(x[(count - 1) / 2], x[count / 2]);
    const REAL right_x = F(midpoint)(x[m - count + (count - 1) / 2], x[m - count + count / 2]);
    const REAL slope = paired ? (right_level - left_level) / (right_x - left_x) : (REAL)0;
    const REAL level = paired ? left_level : *baseline;
    if (!ISFINR(slope))
        return 1;
    for (size_t j = 0; j < m; ++j) {
        signal[j] = y[j] - (level + slope * (x[j] - left_x));
        if (!ISFINR(signal[j]))
            return 1;
    }
    for (size_t j = 0; j < count; ++j) {
        edges[j] = FABSR(y[j] - left_level);
        edges[count + j] = FABSR(y[m - count + j] - right_level);
    }
    const REAL noise = (REAL)1.4826 * F(median)(edges, 2 * count);
    if (!ISFINR(noise))
        return 1;
    size_t first = m;
    REAL height = 0;
    for (size_t j = 1; j + 1 < m; ++j) {
        const REAL value = F(smooth)(signal, m, j);
        if (value > height && value > F(smooth)(signal, m, j - 1) &&
            value >= F(smooth)(signal, m, j + 1)) {
            first = j;
            height = value;
        }
    }
    if (first == m || height <= (REAL)3 * noise)
        return 2;
    first = F(raw_maximum)(signal, first);
    F(peak_t) primary = F(peak)(x, signal, m, first, 0, m - 1, 0);
    if (!primary.valid)
        return 2;
    if (!paired) {
        params[0] = primary.amplitude;
        params[1] = primary.center;
        if (model == 0)
            params[2] = primary.width / (REAL)2.354820045030949382;
        else if (model == 1)
            params[2] = primary.width / (REAL)2;
        else {
            params[2] = primary.width;
            params[3] = (REAL)0.5;
        }
    } else {
        const REAL separation = F(maxr)((REAL)3 * spacing,
                                        (REAL)2 * F(minr)(primary.left_radius,
                                                          primary.right_radius));
        size_t second = m;
        REAL second_height = 0;
        for (size_t j = 1; j + 1 < m; ++j) {
            const REAL value = F(smooth)(signal, m, j);
            if (value <= second_height || value <= F(smooth)(signal, m, j - 1) ||
                value < F(smooth)(signal, m, j + 1))
                continue;
            const size_t index = F(raw_maximum)(signal, j);
            const size_t bins = index > first ? index - first : first - index;
            if (bins < 3 || FABSR(x[index] - primary.center) < separation ||
                F(prominence)(signal, m, j) <= (REAL)3 * noise)
                continue;
            second = index;
            second_height = value;
        }
        if (second == m)
            return 3;
        if (first > second) {
            const size_t t = first;
            first = second;
            second = t;
        }
        size_t valley = first + 1;
        for (size_t j = first + 2; j < second; ++j)
            if (signal[j] < signal[valley])
                valley = j;
        primary = F(peak)(x, signal, m, first, 0, valley, 1);
        const F(peak_t) secondary = F(peak)(x, signal, m, second, valley, m - 1, 1);
        if (!primary.valid || !secondary.valid || !(primary.center < secondary.center))
            return 3;
        params[0] = primary.amplitude;
        params[1] = primary.center;
        params[2] = primary.width / (REAL)2;
        params[3] = secondary.amplitude;
        params[4] = secondary.center;
        params[5] = secondary.width / (REAL)2;
        params[6] = left_level - slope * left_x;
        params[7] = slope;
    }
    for (unsigned k = 0; k < p; ++k)
        if (!ISFINR(params[k]))
            return 1;
    if (!(params[2] > (REAL)0) || (paired && !(params[5] > (REAL)0)))
        return 1;
    return 0;
}

int F(bfo_guess)(int model, size_t n, size_t m, const REAL *x, const REAL *y, REAL *params,
                 int32_t *gstatus, REAL *baseline) {
    if (model < 0 || model > 3)
        return 1;
    const unsigned p = bfo_pcount(model);
    const size_t count = m / 10 > 1 ? m / 10 : 1;
    REAL *edges = (REAL *)malloc(sizeof(REAL) * (2 * count + m + 1));
    if (!edges)
        return 2;
    REAL *signal = edges + 2 * count;
    for (size_t i = 0; i < n; ++i) {
        REAL base;
        const int32_t s =
            F(guess_one)(model, x, y + i * m, m, params + i * p, &base, edges, signal);
        if (gstatus)
            gstatus[i] = s;
        if (baseline)
            baseline[i] = base;
    }
    free(edges);
    return 0;
}

/* cpu::fit_batch (include/batchfit/cpu/batch.hpp:23-65) with the Python binding's
 * p0=None guesses (python/bindings.cpp:69-80); serial. */
int F(bfo_fit)(int model, size_t n, size_t m, const REAL *x, const REAL *y, const REAL *p0,
               const REAL *lower, const REAL *upper, const bfo_options *options,
               int uncertainties, REAL *params, int32_t *status, uint32_t *iterations,
               REAL *chi2, REAL *covariance, REAL *stderr_out, int32_t *ustatus,
               bfo_counters *counters) {
    if (!bfo_known(model) || (!p0 && !bfo_spectral(model)))
        return 1;
    const unsigned p = bfo_pcount(model);
    F(opts) o;
    o.max_iterations = 100;
    o.lambda0 = (REAL)1e-3;
    o.gtol = sizeof(REAL) == 4 ? (REAL)1e-5 : (REAL)1e-10;
    o.xtol = sizeof(REAL) == 4 ? (REAL)1e-6 : (REAL)1e-10;
    o.ftol = sizeof(REAL) == 4 ? (REAL)1e-6 : (REAL)1e-12;
    o.compensated = 0;
    o.scaled = 0;
    if (options && options->set) {
        o.max_iterations = options->max_iterations;
        o.lambda0 = (REAL)options->initial_lambda;
        o.gtol = (REAL)options->gradient_tolerance;
        o.xtol = (REAL)options->step_tolerance;
        o.ftol = (REAL)options->cost_tolerance;
        o.compensated = options->compensated_sum != 0;
        o.scaled = options->scaled_cholesky != 0;
    }
    for (unsigned k = 0; k < p; ++k) {
        o.lo[k] = lower[k];
        o.hi[k] = upper[k];
    }
    const size_t count = m / 10 > 1 ? m / 10 : 1;
    REAL *scratch = (REAL *)malloc(sizeof(REAL) * (2 * count + m + 1));
    if (!scratch)
        return 2;
    for (size_t i = 0; i < n; ++i) {
        REAL initial[8];
        if (p0) {
            for (unsigned k = 0; k < p; ++k)
                initial[k] = p0[i * p + k];
        } else {
            REAL base;
            F(guess_one)(model, x, y + i * m, m, initial, &base, scratch, scratch + 2 * count);
        }
        status[i] = F(fit_single)(model, p, x, y + i * m, m, initial, &o, params + i * p,
                                  &iterations[i], &chi2[i], counters);
        if (counters)
            counters->iterations += iterations[i];
        if (uncertainties)
            ustatus[i] = F(uncertainty)(model, p, x, m, params + i * p, status[i], chi2[i],
                                        o.lo, o.hi, covariance + i * p * p, stderr_out + i * p);
    }
    free(scratch);
    return 0;
}
