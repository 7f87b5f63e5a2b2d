// Bounded Levenberg-Marquardt for one spectrum per thread group.
//
// Semantics follow cpu::fit_single (include/batchfit/cpu/solver.hpp:195-342) and
// cpu::estimate_uncertainty (include/batchfit/cpu/uncertainty.hpp:12-110):
// preflight, projection, degenerate-data diagnosis, active set, damped Cholesky,
// gain-ratio damping update, the three stop rules and all six statuses.
//
// The B200 arrangement:
//  * one fused pass per trial point evaluates chi2, J^T r and J^T J together
//    (FP32 model/Jacobian, per-lane FP32 partial sums, two-sum reduce-scatter
//    across the group, results as FP64 in shared memory).  A rejected trial
//    leaves the accepted state untouched, so the reference's re-linearisation at
//    an unchanged point is never recomputed;
//  * every group lane runs the P x P control redundantly in FP64 (damped
//    Cholesky, predicted reduction, gain ratio, lambda) -- no broadcasts needed;
//  * the information matrix for the covariance is the accepted state's J^T J,
//    inverted in FP64 (one factorisation, P triangular solves).
#pragma once

#include "bf_args.h"
#include <cuda_fp16.h>
#include "bf_device.cuh"
#include "bf_guess.cuh"
#include "bf_models.cuh"

namespace bf {

enum FitStatus : int {
    kConverged = 0,
    kMaxIterations = 1,
    kSingular = 2,
    kInvalid = 3,
    kDegenerate = 4,
    kUnresolved = 5
};
enum UncertaintyStatus : int {
    kAvailable = 0,
    kNotConverged = 1,
    kInsufficientDof = 2,
    kUSingular = 3,
    kActiveBound = 4,
    kUInvalid = 5
};

constexpr double kFltEps = 1.1920928955078125e-07;
constexpr double kDblEps = 2.220446049250313080847e-16;

template <int MODEL> struct Layout {
    static constexpr int P = Model<MODEL>::P;
    static constexpr int K = 1 + P + P * (P + 1) / 2; // chi2, g[P], lower(A)
    static constexpr int KP = pow2ceil(K);
    __host__ __device__ static constexpr int tri(int k, int l) { return 1 + P + k * (k + 1) / 2 + l; }
};

// Point pairs a lane evaluates between two folds of chi2 and J^T r into its
// compensated running sums: each half of a pair accumulator sums that many points
// naively (the even or the odd points of the lane's run).  Measured on B200 (1M
// pseudo-Voigt fits, M=512; 262,144 two-Lorentzian spectra, M=1024): 4 pairs for the
// 3- and 4-parameter models, 2 for the two-Lorentzian, whose 8-parameter pass holds
// more live values per pair.
template <int MODEL> constexpr int lm_pairs() { return Model<MODEL>::P <= 4 ? 4 : 2; }

// One fused pass at parameters p: state[0] = chi2, state[1..P] = J^T r,
// state[tri(k,l)] = (J^T J)_kl, as FP64 values.
//
// Evaluation: each lane takes two adjacent points at a time and evaluates them with
// packed float32 pairs (sm_100 f32x2: one instruction, two IEEE results), so the
// model, the residual and every accumulation cost half the issue slots of scalar
// code.  Lane `lane` of LANES takes the pairs starting at 2 lane, 2 (lane + LANES),
// ...  PAIRED_LOADS: xs and ys are 8-byte aligned (shared-memory copies, or aligned
// global rows) and a pair is read with one load; otherwise point by point.  Both
// give identical results.
//
// Accumulation: the pair accumulators of a lane sum a few pairs naively; the two
// halves are then added and folded into Kahan pairs for chi2 and J^T r
// (numerics::add, numerics.hpp:12-18).  J^T r decides where the iteration stops
// (its error moves the fixed point), so its per-lane sums are compensated; J^T J
// only shapes the step and sums each lane's pairs naively (at most M / 2G points
// per accumulator).  All of them then enter one two-sum reduce-scatter across the
// lanes (J^T J with zero low parts), so every cross-lane addition is compensated.
// For P <= 4, J^T J is summed in pairs too (2 T registers); the 8-parameter model
// keeps scalar sums of its 36 J^T J terms, which would not fit the registers twice.
//
// pass_sums leaves a lane's partial sums in hi/lo (value hi + lo): slot 0 chi2,
// slots 1..P J^T r, slots KC.. the J^T J lower triangle; slots past KC + T are zero.
template <int MODEL, int LANES, bool PAIRED_LOADS, int KP>
__device__ __forceinline__ void pass_sums(int lane, const float *xs, const float *ys, int m, const float *p,
                                          float (&hi)[KP], float (&lo)[KP]) {
    constexpr int P = Model<MODEL>::P;
    constexpr int KC = P + 1;          // chi2 and J^T r
    constexpr int T = P * (P + 1) / 2; // J^T J lower triangle
    constexpr bool kPairedA = P <= 4;
    constexpr int kPairs = lm_pairs<MODEL>();
    static_assert(KP >= KC + T, "slot arrays");
    const auto q = Model<MODEL>::prepare2(p);
    float2 aa2[kPairedA ? T : 1];
#pragma unroll
    for (int i = 0; i < KP; ++i) {
        hi[i] = 0.0f;
        lo[i] = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < (kPairedA ? T : 1); ++i)
        aa2[i] = splat2(0.0f);
    // Points j and j + 1 (j even); `second` false: j + 1 is past the end -- it is not
    // read, and the pair's second half adds nothing.  xs and ys may be shared or
    // global memory: generic loads only.
    auto load = [&](int j, bool second, float2 &xv, float2 &yv) {
        if (PAIRED_LOADS && second) {
            xv = *reinterpret_cast<const float2 *>(xs + j);
            yv = *reinterpret_cast<const float2 *>(ys + j);
        } else {
            xv.x = xs[j];
            yv.x = ys[j];
            xv.y = second ? xs[j + 1] : xv.x;
            yv.y = second ? ys[j + 1] : yv.x;
        }
    };
    auto pair = [&](float2 xv, float2 yv, bool second, float2 (&part)[KC]) {
        float2 J[P];
        float2 r = Model<MODEL>::residual2(q, xv, yv, J);
        if (!second) {
            r.y = 0.0f;
#pragma unroll
            for (int k = 0; k < P; ++k)
                J[k].y = 0.0f;
        }
        part[0] = fma2(r, r, part[0]);
#pragma unroll
        for (int k = 0; k < P; ++k) {
            part[1 + k] = fma2(J[k], r, part[1 + k]);
#pragma unroll
            for (int l = 0; l <= k; ++l) {
                const int t = k * (k + 1) / 2 + l;
                if constexpr (kPairedA) {
                    aa2[t] = fma2(J[k], J[l], aa2[t]);
                } else {
                    hi[KC + t] = fmaf(J[k].x, J[l].x, hi[KC + t]);
                    hi[KC + t] = fmaf(J[k].y, J[l].y, hi[KC + t]);
                }
            }
        }
    };
    // Kahan fold of both halves; lo holds minus the Kahan correction, so the value is hi + lo.
    auto fold = [&](const float2 (&part)[KC]) {
#pragma unroll
        for (int i = 0; i < KC; ++i) {
            const float adjusted = __fadd_rn(__fadd_rn(part[i].x, part[i].y), lo[i]);
            const float next = __fadd_rn(hi[i], adjusted);
            lo[i] = __fsub_rn(adjusted, __fsub_rn(next, hi[i]));
            hi[i] = next;
        }
    };
    // Full runs of kPairs pairs per lane without bounds checks, then one masked tail.
    constexpr int span = 2 * LANES * kPairs;
    const int full = m - m % span;
    for (int base = 2 * lane; base < full; base += span) {
        float2 part[KC];
#pragma unroll
        for (int i = 0; i < KC; ++i)
            part[i] = splat2(0.0f);
#pragma unroll
        for (int c = 0; c < kPairs; ++c) {
            float2 xv, yv;
            load(base + 2 * LANES * c, true, xv, yv);
            pair(xv, yv, true, part);
        }
        fold(part);
    }
    if (full < m) {
        float2 part[KC];
#pragma unroll
        for (int i = 0; i < KC; ++i)
            part[i] = splat2(0.0f);
#pragma unroll
        for (int c = 0; c < kPairs; ++c) {
            const int j = full + 2 * lane + 2 * LANES * c;
            if (j < m) {
                const bool second = j + 1 < m;
                float2 xv, yv;
                load(j, second, xv, yv);
                pair(xv, yv, second, part);
            }
        }
        fold(part);
    }
    if constexpr (kPairedA) {
#pragma unroll
        for (int t = 0; t < T; ++t)
            hi[KC + t] = __fadd_rn(aa2[t].x, aa2[t].y);
    }
}

// The pass of one group: the group's lanes reduce their sums into `state`.
// Returns whether every sum is finite (the reference's linearize() check,
// solver.hpp:182-190, plus chi2).
template <int MODEL, int G, bool PAIRED_LOADS>
__device__ __forceinline__ bool lm_pass(const Group<G> &g, const float *xs, const float *ys, int m,
                                        const float *p, double *state) {
    constexpr int K = Layout<MODEL>::K;
    constexpr int KP = reduce_slots(K, G);
    float hi[KP], lo[KP];
    pass_sums<MODEL, G, PAIRED_LOADS>(int(g.lane), xs, ys, m, p, hi, lo);
    bool finite = reduce_scatter_store<G, KP>(g, hi, lo, state, K);
    finite = g.all(finite);
    g.sync();
    return finite;
}

// In-place Cholesky of a packed lower triangle (FP64) and solve of rhs.
// Mirrors detail::cholesky_solve (solver.hpp:98-143): the optional diagonal
// equilibration and every finiteness/positivity rejection.  Pivots use rsqrt
// (one reciprocal square root instead of a root and a division), and a failure
// is recorded in a flag instead of an early return, so the groups of a warp do
// not diverge inside the factorisation; the result is only used when it is true.
template <int P>
__device__ __forceinline__ bool chol_solve(double (&a)[P * (P + 1) / 2], double (&b)[P], bool scaled) {
    auto at = [](int i, int j) { return i * (i + 1) / 2 + j; };
    bool ok = true;
    double sinv[P];
    if (scaled) {
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const double d = a[at(i, i)];
            ok = ok & isfinite(d) & (d > 0.0);
            sinv[i] = rsqrt(d);
        }
#pragma unroll
        for (int i = 0; i < P; ++i) {
            b[i] *= sinv[i];
#pragma unroll
            for (int j = 0; j <= i; ++j)
                a[at(i, j)] = (a[at(i, j)] * sinv[i]) * sinv[j];
        }
    }
    double inv[P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double v = a[at(i, j)];
#pragma unroll
            for (int k = 0; k < j; ++k)
                v -= a[at(i, k)] * a[at(j, k)];
            ok = ok & isfinite(v);
            if (i == j) {
                ok = ok & (v > 0.0);
                inv[i] = rsqrt(v);
                a[at(i, i)] = v * inv[i];
            } else {
                a[at(i, j)] = v * inv[j];
            }
        }
        double v = b[i];
#pragma unroll
        for (int j = 0; j < i; ++j)
            v -= a[at(i, j)] * b[j];
        b[i] = v * inv[i];
    }
#pragma unroll
    for (int i = P - 1; i >= 0; --i) {
        double v = b[i];
#pragma unroll
        for (int j = i + 1; j < P; ++j)
            v -= a[at(j, i)] * b[j];
        b[i] = v * inv[i];
        ok = ok & isfinite(b[i]);
    }
    if (scaled) {
#pragma unroll
        for (int i = 0; i < P; ++i) {
            b[i] *= sinv[i];
            ok = ok & isfinite(b[i]);
        }
    }
    return ok;
}

// free_shape (solver.hpp:70-82).
template <int MODEL> __device__ __forceinline__ bool free_shape(const FitArgs &a) {
    bool free = a.lower[1] != a.upper[1] || a.lower[2] != a.upper[2];
    if constexpr (MODEL == kPseudoVoigt)
        free = free || a.lower[3] != a.upper[3];
    if constexpr (MODEL == kTwoLorentzian)
        free = free || a.lower[4] != a.upper[4] || a.lower[5] != a.upper[5];
    return free;
}

// spectral_success (solver.hpp:83-96).
template <int MODEL> __device__ __forceinline__ int spectral_success(const float *p, float spacing) {
    constexpr float factor = Model<MODEL>::width_factor;
    if (spacing > 0.0f && fabsf(p[2]) * factor < spacing)
        return kUnresolved;
    if constexpr (MODEL == kTwoLorentzian)
        if (spacing > 0.0f && fabsf(p[5]) * factor < spacing)
            return kUnresolved;
    return kConverged;
}

// Per-fit LM state carried between rounds (registers).  The accepted J^T J, J^T r
// and chi2 live in shared-memory slot `cur`; a pass writes slot 1 - cur.
template <int MODEL> struct LmState {
    static constexpr int P = Model<MODEL>::P;
    float p[P];       // accepted parameters (reported)
    float t[P];       // point of the next pass: the projected initial values or a trial
    double chi2;      // accepted objective
    double lambda, lambda_max, predicted;
    uint32_t it;         // iteration index (solver.hpp:254)
    uint32_t iterations; // reported attempted updates (solver.hpp:287)
    int status;
    int cur;
    bool initial;    // the next pass is the fit's initial cost + linearisation
    bool cur_finite; // the accepted slot's chi2, J^T r and J^T J are all finite
};

// Start a fit whose inputs passed preflight: project the initial values into the
// bounds (solver.hpp:227-229); the first pass evaluates there.
template <int MODEL> __device__ __forceinline__ void lm_begin(const FitArgs &a, LmState<MODEL> &s) {
#pragma unroll
    for (int k = 0; k < Model<MODEL>::P; ++k) {
        s.p[k] = sclamp(s.p[k], a.lower[k], a.upper[k]);
        s.t[k] = s.p[k];
    }
    s.initial = true;
    s.cur = 0;
    s.it = 0;
    s.iterations = 0;
    s.status = kMaxIterations;
}

// Consume the pass that just wrote slot 1 - s.cur.  Returns true when the fit is
// finished (s.status final).
template <int MODEL, class Grp>
__device__ __forceinline__ bool lm_after_pass(const Grp &g, const FitArgs &a, const XConst &xc, bool y_flat,
                                              bool pass_finite, const double *state, LmState<MODEL> &s) {
    using L = Layout<MODEL>;
    const double c = state[(1 - s.cur) * L::K];
    if (s.initial) {
        // Initial cost and linearisation (solver.hpp:230-253).
        s.initial = false;
        if (!isfinite(c)) {
            s.status = kInvalid;
            s.chi2 = __longlong_as_double(0x7ff8000000000000ll);
            return true;
        }
        s.chi2 = c;
        if (xc.varied_x && y_flat && free_shape<MODEL>(a)) {
            s.status = kDegenerate;
            return true;
        }
        s.cur = 1 - s.cur;
        s.cur_finite = pass_finite;
        s.lambda = a.lambda0;
        s.lambda_max = fmax(a.lambda0, 1.0 / kFltEps);
        return false;
    }
    // Accept / reject the trial and update lambda (solver.hpp:313-339).
    const double reduction = s.chi2 - c;
    const double threshold = a.ftol * s.chi2;
    const bool small = isfinite(c) && isfinite(s.predicted) && s.predicted >= 0.0 && fabs(reduction) <= threshold &&
                       s.predicted <= threshold / fmax(1.0, s.lambda);
    if (isfinite(c) && reduction > 0.0 && isfinite(s.predicted) && s.predicted > 0.0) {
#pragma unroll
        for (int k = 0; k < Model<MODEL>::P; ++k)
            s.p[k] = s.t[k];
        s.chi2 = c;
        s.cur = 1 - s.cur;
        s.cur_finite = pass_finite;
        const double ratio = reduction / s.predicted;
        const double u = 2.0 * ratio - 1.0;
        const double factor = ratio >= 1.0 ? 1.0 / 3.0 : fmax(1.0 / 3.0, 1.0 - u * u * u);
        s.lambda = dclamp(s.lambda * factor, a.policy == kPolicyParity ? kDblEps : kFltEps, s.lambda_max);
    } else {
        s.lambda = fmin(s.lambda_max, s.lambda * 10.0);
    }
    // The next pass overwrites the slot just read.
    g.sync();
    s.it += 1;
    if (small) {
        s.status = spectral_success<MODEL>(s.p, xc.spacing);
        return true;
    }
    return false;
}

// Plan the next trial from the accepted state (solver.hpp:254-312).  Returns true
// when the fit finished instead; otherwise s.t holds the next pass point.
template <int MODEL>
__device__ __forceinline__ bool lm_plan(const FitArgs &a, const XConst &xc, double syy, const double *state,
                                        LmState<MODEL> &s) {
    using L = Layout<MODEL>;
    constexpr int P = L::P;
    const bool parity = a.policy == kPolicyParity;
    while (true) {
        if (s.it >= a.max_iterations)
            return true; // status stays max_iterations
        const double *cur = state + s.cur * L::K;
        const double *A = cur + 1 + P; // packed lower triangle
        const double *gr = cur + 1;
        if (!s.cur_finite) {
            s.status = kInvalid;
            return true;
        }
        bool active[P];
        double gnorm = 0.0;
        bool at_floor = true;
        // |g_k| <= floor * eps * sqrt(A_kk * sum(y^2)), compared squared (both sides
        // are non-negative), so the control takes no square roots.
        const double floor_e = a.noise_floor * kFltEps;
        const double floor2 = floor_e * floor_e * syy;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const double gk = gr[k];
            active[k] = a.lower[k] == a.upper[k] || (s.p[k] == a.lower[k] && gk < 0.0) ||
                        (s.p[k] == a.upper[k] && gk > 0.0);
            if (!active[k]) {
                gnorm = fmax(gnorm, fabs(gk));
                at_floor = at_floor && gk * gk <= floor2 * fmax(A[k * (k + 1) / 2 + k], 0.0);
            }
        }
        if (gnorm <= a.gtol || (parity && at_floor)) {
            s.status = spectral_success<MODEL>(s.p, xc.spacing);
            return true;
        }
        double D[P * (P + 1) / 2], delta[P];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            delta[k] = active[k] ? 0.0 : gr[k];
#pragma unroll
            for (int l = 0; l <= k; ++l) {
                double v = A[k * (k + 1) / 2 + l];
                if (active[k] || active[l])
                    v = 0.0;
                if (k == l)
                    v = active[k] ? 1.0 : v + s.lambda * A[k * (k + 1) / 2 + k];
                D[k * (k + 1) / 2 + l] = v;
            }
        }
        s.iterations = s.it + 1;
        if (!chol_solve<P>(D, delta, (a.flags & kFlagScaledCholesky) != 0u)) {
            s.status = kSingular;
            return true;
        }
        double step_norm = 0.0, param_norm = 0.0;
        bool finite_trial = true;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            step_norm = fmax(step_norm, fabs(delta[k]));
            s.t[k] = float(dclamp(double(s.p[k]) + delta[k], double(a.lower[k]), double(a.upper[k])));
            finite_trial = finite_trial && isfinite(s.t[k]);
            delta[k] = double(s.t[k]) - double(s.p[k]);
            param_norm = fmax(param_norm, fabs(double(s.p[k])));
        }
        const double damp = fmax(1.0, s.lambda);
        if (step_norm <= a.xtol * (param_norm + a.xtol) / damp ||
            (parity && step_norm * damp <= a.step_quantum * kFltEps * param_norm)) {
            s.status = spectral_success<MODEL>(s.p, xc.spacing);
            return true;
        }
        double predicted = 0.0;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            predicted += 2.0 * gr[k] * delta[k];
#pragma unroll
            for (int l = 0; l < P; ++l) {
                const double akl = k >= l ? A[k * (k + 1) / 2 + l] : A[l * (l + 1) / 2 + k];
                predicted -= delta[k] * akl * delta[l];
            }
        }
        s.predicted = predicted;
        if (finite_trial)
            return false;
        // A non-finite trial has a NaN cost: rejected without evaluation.
        s.lambda = fmin(s.lambda_max, s.lambda * 10.0);
        s.it += 1;
    }
}

// Covariance of one converged fit (include/batchfit/cpu/uncertainty.hpp:12-110),
// one thread per fit.  `info` holds the accepted state's J^T J (P*P floats, the LM
// kernel writes it into the caller's covariance output); it is replaced by the
// covariance.  The inverse is FP64: one equilibrated Cholesky factorisation and P
// triangular solves (the reference refactors per column with the same result).
template <int MODEL>
__device__ int covariance_one(const FitArgs &a, const float *p, int fit_status, float chi2f, float *info,
                              float *se_out) {
    constexpr int P = Model<MODEL>::P;
    const float qnan = __int_as_float(0x7fffffff);
    int status = kAvailable;
    bool fixed[P];
    int nfree = 0;
    if (fit_status != kConverged)
        status = kNotConverged;
    else if (!isfinite(chi2f) || chi2f < 0.0f)
        status = kUInvalid;
#pragma unroll
    for (int k = 0; k < P; ++k) {
        fixed[k] = a.lower[k] == a.upper[k];
        nfree += fixed[k] ? 0 : 1;
        if (status != kAvailable)
            continue;
        if (!isfinite(p[k]) || isnan(a.lower[k]) || isnan(a.upper[k]) || a.lower[k] > a.upper[k] ||
            p[k] < a.lower[k] || p[k] > a.upper[k])
            status = kUInvalid;
        else if (!fixed[k] && (p[k] == a.lower[k] || p[k] == a.upper[k]))
            status = kActiveBound;
    }
    if (status == kAvailable && a.m <= nfree)
        status = kInsufficientDof;
    double H[P * (P + 1) / 2];
    double inv[P];
    if (status == kAvailable) {
#pragma unroll
        for (int k = 0; k < P; ++k)
#pragma unroll
            for (int l = 0; l <= k; ++l) {
                double v = double(info[k * P + l]);
                if (!isfinite(v))
                    status = kUInvalid;
                if (fixed[k] || fixed[l])
                    v = (k == l) ? 1.0 : 0.0;
                H[k * (k + 1) / 2 + l] = v;
            }
    }
    const double variance = double(chi2f) / double(a.m - nfree);
    if (status == kAvailable && !isfinite(variance))
        status = kUInvalid;
    if (status == kAvailable) {
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const double d = H[i * (i + 1) / 2 + i];
            if (!isfinite(d) || d <= 0.0)
                status = kUSingular;
            inv[i] = rsqrt(d);
        }
    }
    if (status == kAvailable) {
#pragma unroll
        for (int i = 0; i < P; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j)
                H[i * (i + 1) / 2 + j] = H[i * (i + 1) / 2 + j] * inv[i] * inv[j];
        const double pivot_floor = 64.0 * (a.policy == kPolicyParity ? kDblEps : kFltEps);
        double linv[P];
#pragma unroll
        for (int i = 0; i < P; ++i) {
#pragma unroll
            for (int j = 0; j <= i; ++j) {
                double v = H[i * (i + 1) / 2 + j];
#pragma unroll
                for (int k = 0; k < j; ++k)
                    v -= H[i * (i + 1) / 2 + k] * H[j * (j + 1) / 2 + k];
                if (!isfinite(v) || (i == j && v <= 0.0))
                    status = kUSingular;
                if (i == j) {
                    linv[i] = rsqrt(v);
                    H[i * (i + 1) / 2 + i] = v * linv[i];
                } else {
                    H[i * (i + 1) / 2 + j] = v * linv[j];
                }
            }
        }
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (!fixed[i] && H[i * (i + 1) / 2 + i] * H[i * (i + 1) / 2 + i] <= pivot_floor)
                status = kUSingular;
        if (status == kAvailable) {
            // Column `column` of the inverse into info[.. * P + column].
#pragma unroll
            for (int column = 0; column < P; ++column) {
                double b[P];
#pragma unroll
                for (int i = 0; i < P; ++i)
                    b[i] = (i == column) ? inv[i] : 0.0;
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    double v = b[i];
#pragma unroll
                    for (int j = 0; j < i; ++j)
                        v -= H[i * (i + 1) / 2 + j] * b[j];
                    b[i] = v * linv[i];
                }
#pragma unroll
                for (int i = P - 1; i >= 0; --i) {
                    double v = b[i];
#pragma unroll
                    for (int j = i + 1; j < P; ++j)
                        v -= H[j * (j + 1) / 2 + i] * b[j];
                    b[i] = v * linv[i];
                }
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    const double c = fixed[column] || fixed[i] ? 0.0 : (b[i] * inv[i]) * variance;
                    if (!isfinite(c))
                        status = kUInvalid;
                    info[i * P + column] = float(c);
                }
            }
        }
    }
    // Symmetrise (uncertainty.hpp:96-103) or publish NaN on any failure.
    if (status == kAvailable) {
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (info[i * P + i] < 0.0f)
                status = kUInvalid;
    }
    if (status == kAvailable) {
#pragma unroll
        for (int i = 0; i < P; ++i)
#pragma unroll
            for (int j = 0; j < i; ++j) {
                const float v = info[i * P + j] / 2.0f + info[j * P + i] / 2.0f;
                info[i * P + j] = v;
                info[j * P + i] = v;
            }
#pragma unroll
        for (int i = 0; i < P; ++i)
            se_out[i] = sqrtf(info[i * P + i]);
    } else {
#pragma unroll
        for (int k = 0; k < P * P; ++k)
            info[k] = qnan;
#pragma unroll
        for (int i = 0; i < P; ++i)
            se_out[i] = qnan;
    }
    return status;
}

// Outputs of a finished fit (FitResult, solver.hpp:43-48).
template <int MODEL, class Grp>
__device__ __forceinline__ void write_fit(const Grp &g, const FitArgs &a, long long fit, const LmState<MODEL> &s) {
    constexpr int P = Model<MODEL>::P;
#pragma unroll
    for (int k = 0; k < P; ++k)
        if (int(g.lane) == k)
            a.params[fit * P + k] = s.p[k];
    if (g.lane == 0) {
        a.status[fit] = s.status;
        a.iterations[fit] = s.iterations;
        a.chi2[fit] = float(s.chi2);
    }
}

// The accepted J^T J (the information matrix at the reported parameters), left in
// the covariance output for the covariance kernel.
template <int MODEL, class Grp>
__device__ __forceinline__ void write_information(const Grp &g, const FitArgs &a, long long fit,
                                                  const double *cur) {
    constexpr int P = Model<MODEL>::P;
    for (int k = int(g.lane); k < P * P; k += Grp::size) {
        const int i = k / P, j = k % P;
        a.covariance[fit * P * P + k] = float(cur[Layout<MODEL>::tri(i > j ? i : j, i > j ? j : i)]);
    }
}

// Stage one fit-major y row into shared memory (kStore) or only scan it; reports
// finiteness and, with kSums, flatness (every value equal to y[0]) and sum(y^2),
// with the same arithmetic either way (without kSums: flat false, syy 0).
template <int G, bool kStore = true, bool kSums = true>
__device__ __forceinline__ void stage_row(const Group<G> &g, const float *row, int m, bool vec_ok, float *ys,
                                          bool &yfin, bool &flat, float &syy) {
    const float y0 = __ldg(row);
    yfin = true;
    flat = true;
    syy = 0.0f;
    if (vec_ok) {
        const float4 *row4 = reinterpret_cast<const float4 *>(row);
        for (int v = int(g.lane); v < m / 4; v += G) {
            const float4 t = kStore ? __ldcs(row4 + v) : __ldg(row4 + v);
            if constexpr (kStore)
                reinterpret_cast<float4 *>(ys)[v] = t;
            yfin = yfin && isfinite(t.x) && isfinite(t.y) && isfinite(t.z) && isfinite(t.w);
            if constexpr (kSums) {
                flat = flat && t.x == y0 && t.y == y0 && t.z == y0 && t.w == y0;
                syy = fmaf(t.x, t.x, fmaf(t.y, t.y, fmaf(t.z, t.z, fmaf(t.w, t.w, syy))));
            }
        }
    } else {
        for (int j = int(g.lane); j < m; j += G) {
            const float t = kStore ? __ldcs(row + j) : __ldg(row + j);
            if constexpr (kStore)
                ys[j] = t;
            yfin = yfin && isfinite(t);
            if constexpr (kSums) {
                flat = flat && t == y0;
                syy = fmaf(t, t, syy);
            }
        }
    }
    yfin = g.all(yfin);
    if constexpr (kSums) {
        flat = g.all(flat);
#pragma unroll
        for (int o = G / 2; o >= 1; o >>= 1)
            syy += g.xor_(syy, o);
    } else {
        flat = false;
    }
    g.sync();
}

// A row of y stored as IEEE binary16 (opt-in half-precision storage), converted
// exactly to float32 while it is staged, with stage_row's accumulations in the same
// order: a fit of half-precision y equals the fit of the same values given as float.
template <int G, bool kSums = true>
__device__ __forceinline__ void stage_row_half(const Group<G> &g, const __half *row, int m, bool vec_ok, float *ys,
                                               bool &yfin, bool &flat, float &syy) {
    const float y0 = __half2float(row[0]);
    yfin = true;
    flat = true;
    syy = 0.0f;
    if (vec_ok) {
        const uint2 *row4 = reinterpret_cast<const uint2 *>(row);
        for (int v = int(g.lane); v < m / 4; v += G) {
            const uint2 raw = __ldcs(row4 + v);
            const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&raw.x));
            const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&raw.y));
            const float4 t = make_float4(a.x, a.y, b.x, b.y);
            reinterpret_cast<float4 *>(ys)[v] = t;
            yfin = yfin && isfinite(t.x) && isfinite(t.y) && isfinite(t.z) && isfinite(t.w);
            if constexpr (kSums) {
                flat = flat && t.x == y0 && t.y == y0 && t.z == y0 && t.w == y0;
                syy = fmaf(t.x, t.x, fmaf(t.y, t.y, fmaf(t.z, t.z, fmaf(t.w, t.w, syy))));
            }
        }
    } else {
        for (int j = int(g.lane); j < m; j += G) {
            const float t = __half2float(row[j]);
            ys[j] = t;
            yfin = yfin && isfinite(t);
            if constexpr (kSums) {
                flat = flat && t == y0;
                syy = fmaf(t, t, syy);
            }
        }
    }
    yfin = g.all(yfin);
    if constexpr (kSums) {
        flat = g.all(flat);
#pragma unroll
        for (int o = G / 2; o >= 1; o >>= 1)
            syy += g.xor_(syy, o);
    } else {
        flat = false;
    }
    g.sync();
}

// Whether rows of y start 128-bit (float) / 64-bit (half) aligned: 4 values a load.
__device__ __forceinline__ bool rows_vectorisable(const float *y, int m, bool y_half) {
    return (m & 3) == 0 && (reinterpret_cast<uintptr_t>(y) & (y_half ? 7u : 15u)) == 0;
}

// Stage row `fit` of y (float32, or binary16 when y_half) into shared memory.
template <int G, bool kSums = true>
__device__ __forceinline__ void stage_fit_row(const Group<G> &g, const float *y, bool y_half, long long fit, int m,
                                              bool vec_ok, float *ys, bool &yfin, bool &flat, float &syy) {
    if (y_half)
        stage_row_half<G, kSums>(g, reinterpret_cast<const __half *>(y) + fit * m, m, vec_ok, ys, yfin, flat, syy);
    else
        stage_row<G, true, kSums>(g, y + fit * m, m, vec_ok, ys, yfin, flat, syy);
}

// Covariance of one finished fit from the information matrix the LM kernel left in
// its covariance slot: covariance, standard errors and the uncertainty status.
template <int MODEL> __device__ __forceinline__ void covariance_fit(const FitArgs &a, long long fit) {
    constexpr int P = Model<MODEL>::P;
    float p[P], info[P * P], se[P];
#pragma unroll
    for (int k = 0; k < P; ++k)
        p[k] = a.params[fit * P + k];
    const int status = a.status[fit];
    if (status == kConverged) {
#pragma unroll
        for (int k = 0; k < P * P; ++k)
            info[k] = a.covariance[fit * P * P + k];
    }
    const int us = covariance_one<MODEL>(a, p, status, a.chi2[fit], info, se);
#pragma unroll
    for (int k = 0; k < P * P; ++k)
        a.covariance[fit * P * P + k] = info[k];
#pragma unroll
    for (int k = 0; k < P; ++k)
        a.stderr_out[fit * P + k] = se[k];
    a.ustatus[fit] = us;
}

} // namespace bf
