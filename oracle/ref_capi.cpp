// Test infrastructure only: a C ABI over the reference batchfit CPU path, so that
// tests and the CPU-baseline leg of bench.py can call the reference's own
// implementation from Python (ctypes) with plain pointers.  Nothing in the
// batchfit_b200 product links or loads this file's library.
//
// Compiled by oracle/Makefile against the reference headers in place
// (include/batchfit/cpu/{solver,initial_guess,uncertainty,batch}.hpp) and the
// reference's src/cpu/thread_pool.cpp.  The calls below follow the reference
// pybind binding python/bindings.cpp:60-121 (guesses on the pool, then
// cpu::fit_batch) but with a caller-chosen worker count instead of the fixed two.
#include <batchfit/cpu/batch.hpp>
#include <batchfit/cpu/initial_guess.hpp>
#include <batchfit/cpu/solver.hpp>
#include <batchfit/cpu/thread_pool.hpp>
#include <batchfit/cpu/uncertainty.hpp>
#include <batchfit/models.hpp>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <thread>

namespace {
thread_local std::string last_error;

// Mirrors the scalar fields of cpu::SolverOptions (solver.hpp:26-41).  A zero
// `set` means "reference defaults for this scalar type"; bounds always apply.
struct RefOptions {
    uint32_t set;
    uint32_t max_iterations;
    double initial_lambda, gradient_tolerance, step_tolerance, cost_tolerance;
    uint32_t compensated_sum, scaled_cholesky;
};

template <typename T, template <typename> class Model>
batchfit::cpu::SolverOptions<T, Model<T>::parameter_count>
make_options(const RefOptions *in, const T *lower, const T *upper) {
    constexpr unsigned p = Model<T>::parameter_count;
    batchfit::cpu::SolverOptions<T, p> options;
    if (in && in->set) {
        options.max_iterations = in->max_iterations;
        options.initial_lambda = T(in->initial_lambda);
        options.gradient_tolerance = T(in->gradient_tolerance);
        options.step_tolerance = T(in->step_tolerance);
        options.cost_tolerance = T(in->cost_tolerance);
        options.compensated_sum = in->compensated_sum != 0;
        options.scaled_cholesky = in->scaled_cholesky != 0;
    }
    for (unsigned k = 0; k < p; ++k) {
        options.lower[k] = lower[k];
        options.upper[k] = upper[k];
    }
    return options;
}

template <typename T, template <typename> class Model>
int fit_typed(size_t n, size_t m, const T *x, const T *y, const T *p0, const T *lower,
              const T *upper, const RefOptions *opts, int uncertainties, unsigned workers,
              T *params, int32_t *status, uint32_t *iterations, T *chi2, T *covariance,
              T *stderr_out, int32_t *ustatus, double *seconds) {
    constexpr unsigned p = Model<T>::parameter_count;
    batchfit::cpu::ThreadPool pool(workers ? workers : 1);
    const std::span<const T> xs(x, m), ys(y, n * m);
    std::vector<T> generated;
    std::span<const T> initial;
    const auto t0 = std::chrono::steady_clock::now();
    if (p0) {
        initial = std::span<const T>(p0, n * p);
    } else {
        generated.resize(n * p);
        if (n)
            pool.parallel_for(n, [&](size_t begin, size_t end) {
                for (auto i = begin; i < end; ++i) {
                    const auto guess =
                        batchfit::cpu::initial_guess<T, Model>(xs, ys.subspan(i * m, m));
                    std::copy(guess.parameters.begin(), guess.parameters.end(),
                              generated.data() + i * p);
                }
            });
        initial = generated;
    }
    const auto t1 = std::chrono::steady_clock::now();
    const auto options = make_options<T, Model>(opts, lower, upper);
    if (n == 0) {
        if (seconds)
            seconds[0] = seconds[1] = 0;
        return 0;
    }
    const auto result =
        batchfit::cpu::fit_batch<T, Model>(xs, ys, initial, pool, options, uncertainties != 0);
    const auto t2 = std::chrono::steady_clock::now();
    std::memcpy(params, result.parameters.data(), n * p * sizeof(T));
    for (size_t i = 0; i < n; ++i) {
        status[i] = int32_t(result.status[i]);
        iterations[i] = result.iterations[i];
        chi2[i] = result.chi_squared[i];
    }
    if (uncertainties) {
        std::memcpy(covariance, result.covariance.data(), n * p * p * sizeof(T));
        std::memcpy(stderr_out, result.standard_errors.data(), n * p * sizeof(T));
        for (size_t i = 0; i < n; ++i)
            ustatus[i] = int32_t(result.uncertainty_status[i]);
    }
    if (seconds) {
        seconds[0] = std::chrono::duration<double>(t1 - t0).count();
        seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    return 0;
}

template <typename T>
int fit_dispatch(int model, size_t n, size_t m, const void *x, const void *y, const void *p0,
                 const void *lower, const void *upper, const RefOptions *opts, int uncertainties,
                 unsigned workers, void *params, int32_t *status, uint32_t *iterations,
                 void *chi2, void *covariance, void *stderr_out, int32_t *ustatus,
                 double *seconds) {
    const auto *xt = static_cast<const T *>(x);
    const auto *yt = static_cast<const T *>(y);
    const auto *pt = static_cast<const T *>(p0);
    const auto *lo = static_cast<const T *>(lower);
    const auto *hi = static_cast<const T *>(upper);
    auto *pa = static_cast<T *>(params);
    auto *c2 = static_cast<T *>(chi2);
    auto *cv = static_cast<T *>(covariance);
    auto *se = static_cast<T *>(stderr_out);
    switch (model) {
    case 0:
        return fit_typed<T, batchfit::models::Gaussian>(n, m, xt, yt, pt, lo, hi, opts,
                                                        uncertainties, workers, pa, status,
                                                        iterations, c2, cv, se, ustatus, seconds);
    case 1:
        return fit_typed<T, batchfit::models::Lorentzian>(n, m, xt, yt, pt, lo, hi, opts,
                                                          uncertainties, workers, pa, status,
                                                          iterations, c2, cv, se, ustatus, seconds);
    case 2:
        return fit_typed<T, batchfit::models::PseudoVoigt>(n, m, xt, yt, pt, lo, hi, opts,
                                                           uncertainties, workers, pa, status,
                                                           iterations, c2, cv, se, ustatus,
                                                           seconds);
    case 3:
        return fit_typed<T, batchfit::models::TwoLorentzian>(n, m, xt, yt, pt, lo, hi, opts,
                                                             uncertainties, workers, pa, status,
                                                             iterations, c2, cv, se, ustatus,
                                                             seconds);
    default:
        last_error = "unknown model id";
        return 1;
    }
}

template <typename T, template <typename> class Model>
void guess_typed(size_t n, size_t m, const T *x, const T *y, T *params, int32_t *gstatus,
                 T *baseline) {
    constexpr unsigned p = Model<T>::parameter_count;
    const std::span<const T> xs(x, m);
    for (size_t i = 0; i < n; ++i) {
        const auto guess =
            batchfit::cpu::initial_guess<T, Model>(xs, std::span<const T>(y + i * m, m));
        std::copy(guess.parameters.begin(), guess.parameters.end(), params + i * p);
        if (gstatus)
            gstatus[i] = int32_t(guess.status);
        if (baseline)
            baseline[i] = guess.baseline;
    }
}

template <typename T>
int guess_dispatch(int model, size_t n, size_t m, const void *x, const void *y, void *params,
                   int32_t *gstatus, void *baseline) {
    const auto *xt = static_cast<const T *>(x);
    const auto *yt = static_cast<const T *>(y);
    auto *pa = static_cast<T *>(params);
    auto *bl = static_cast<T *>(baseline);
    switch (model) {
    case 0:
        guess_typed<T, batchfit::models::Gaussian>(n, m, xt, yt, pa, gstatus, bl);
        return 0;
    case 1:
        guess_typed<T, batchfit::models::Lorentzian>(n, m, xt, yt, pa, gstatus, bl);
        return 0;
    case 2:
        guess_typed<T, batchfit::models::PseudoVoigt>(n, m, xt, yt, pa, gstatus, bl);
        return 0;
    case 3:
        guess_typed<T, batchfit::models::TwoLorentzian>(n, m, xt, yt, pa, gstatus, bl);
        return 0;
    default:
        last_error = "unknown model id";
        return 1;
    }
}

template <typename T, unsigned P> int cholesky_typed(T *matrix, T *rhs, int scaled) {
    batchfit::cpu::detail::Matrix<T, P> a;
    std::array<T, P> b;
    for (unsigned i = 0; i < P; ++i) {
        b[i] = rhs[i];
        for (unsigned j = 0; j < P; ++j)
            a[i][j] = matrix[i * P + j];
    }
    const bool ok = batchfit::cpu::detail::cholesky_solve<T, P>(a, b, scaled != 0);
    for (unsigned i = 0; i < P; ++i) {
        rhs[i] = b[i];
        for (unsigned j = 0; j < P; ++j)
            matrix[i * P + j] = a[i][j];
    }
    return ok ? 1 : 0;
}

template <typename T> int cholesky_dispatch(unsigned p, void *matrix, void *rhs, int scaled) {
    auto *a = static_cast<T *>(matrix);
    auto *b = static_cast<T *>(rhs);
    switch (p) {
    case 1: return cholesky_typed<T, 1>(a, b, scaled);
    case 2: return cholesky_typed<T, 2>(a, b, scaled);
    case 3: return cholesky_typed<T, 3>(a, b, scaled);
    case 4: return cholesky_typed<T, 4>(a, b, scaled);
    case 8: return cholesky_typed<T, 8>(a, b, scaled);
    default: return -1;
    }
}
} // namespace

extern "C" {
const char *bfref_last_error(void) { return last_error.c_str(); }

unsigned bfref_hardware_concurrency(void) {
    return std::max(1U, std::thread::hardware_concurrency());
}

// dtype: 4 = float32 path (fit_batch<float>), 8 = float64 path (fit_batch<double>).
// p0 == nullptr runs initial_guess<T> per row first, as python/bindings.cpp:69-80.
// seconds[0] = guess wall time, seconds[1] = fit_batch wall time.
int bfref_fit(int model, int dtype, size_t n, size_t m, const void *x, const void *y,
              const void *p0, const void *lower, const void *upper, const RefOptions *opts,
              int uncertainties, unsigned workers, void *params, int32_t *status,
              uint32_t *iterations, void *chi2, void *covariance, void *stderr_out,
              int32_t *ustatus, double *seconds) {
    try {
        if (dtype == 4)
            return fit_dispatch<float>(model, n, m, x, y, p0, lower, upper, opts, uncertainties,
                                       workers, params, status, iterations, chi2, covariance,
                                       stderr_out, ustatus, seconds);
        if (dtype == 8)
            return fit_dispatch<double>(model, n, m, x, y, p0, lower, upper, opts, uncertainties,
                                        workers, params, status, iterations, chi2, covariance,
                                        stderr_out, ustatus, seconds);
        last_error = "dtype must be 4 or 8";
        return 1;
    } catch (const std::exception &error) {
        last_error = error.what();
        return 2;
    }
}

// initial_guess<T,Model> per row (initial_guess.hpp:120-249); serial.
int bfref_guess(int model, int dtype, size_t n, size_t m, const void *x, const void *y,
                void *params, int32_t *gstatus, void *baseline) {
    try {
        if (dtype == 4)
            return guess_dispatch<float>(model, n, m, x, y, params, gstatus, baseline);
        if (dtype == 8)
            return guess_dispatch<double>(model, n, m, x, y, params, gstatus, baseline);
        last_error = "dtype must be 4 or 8";
        return 1;
    } catch (const std::exception &error) {
        last_error = error.what();
        return 2;
    }
}

// cpu::detail::cholesky_solve (solver.hpp:98-143) on a row-major PxP matrix.
int bfref_cholesky_solve(int dtype, unsigned p, void *matrix, void *rhs, int scaled) {
    if (dtype == 4)
        return cholesky_dispatch<float>(p, matrix, rhs, scaled);
    if (dtype == 8)
        return cholesky_dispatch<double>(p, matrix, rhs, scaled);
    return -1;
}
}
