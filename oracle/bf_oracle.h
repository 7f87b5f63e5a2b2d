/* Test infrastructure only: the CPU oracle for the batchfit_b200 CUDA path.
 *
 * A plain-C restatement of the reference batchfit CPU fitting path, used by
 * tests/ (parity checks), __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg.  The product library never links or loads it.
 *
 * Pinned against the compiled reference (oracle/_ref, built from the reference
 * sources by oracle/Makefile) bit for bit on seeded fixtures, and against the
 * known answers of the reference's own tests (tests/golden/).
 *
 * Model ids: 0 gaussian, 1 lorentzian, 2 pseudo_voigt, 3 two_lorentzian
 * (python/batchfit/__init__.py:13), plus the non-spectral models the reference's
 * own known-answer tests use: BFO_LINE p0 + p1*x (tests/uncertainty_checks.hpp:8-15),
 * BFO_CONSTANT p0 (tests/solver_checks.hpp:22-26) and BFO_EXPONENTIAL exp(x*p0)
 * (tests/solver_checks.hpp:27-31).  They have no guess (p0 is required).
 */
#define BFO_LINE 100
#define BFO_CONSTANT 101
#define BFO_EXPONENTIAL 102
#ifndef BF_ORACLE_H
#define BF_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cpu::SolverOptions scalars (include/batchfit/cpu/solver.hpp:26-41).  set == 0
 * selects the reference defaults of the scalar type (float: 1e-5/1e-6/1e-6,
 * double: 1e-10/1e-10/1e-12; 100 iterations; lambda 1e-3). */
typedef struct bfo_options {
    uint32_t set;
    uint32_t max_iterations;
    double initial_lambda, gradient_tolerance, step_tolerance, cost_tolerance;
    uint32_t compensated_sum, scaled_cholesky;
} bfo_options;

/* Per-fit pass counts of the LM trajectory (for the roofline's algorithmic work). */
typedef struct bfo_counters {
    uint64_t cost_passes;      /* detail::cost calls, initial one included */
    uint64_t linearize_passes; /* detail::linearize calls */
    uint64_t iterations;       /* sum of reported iterations */
} bfo_counters;

int bfo_fit_f32(int model, size_t n, size_t m, const float *x, const float *y, const float *p0,
                const float *lower, const float *upper, const bfo_options *options,
                int uncertainties, float *params, int32_t *status, uint32_t *iterations,
                float *chi2, float *covariance, float *stderr_out, int32_t *ustatus,
                bfo_counters *counters);
int bfo_fit_f64(int model, size_t n, size_t m, const double *x, const double *y,
                const double *p0, const double *lower, const double *upper,
                const bfo_options *options, int uncertainties, double *params, int32_t *status,
                uint32_t *iterations, double *chi2, double *covariance, double *stderr_out,
                int32_t *ustatus, bfo_counters *counters);

/* initial_guess<T,Model> (include/batchfit/cpu/initial_guess.hpp:120-249), per row. */
int bfo_guess_f32(int model, size_t n, size_t m, const float *x, const float *y, float *params,
                  int32_t *gstatus, float *baseline);
int bfo_guess_f64(int model, size_t n, size_t m, const double *x, const double *y,
                  double *params, int32_t *gstatus, double *baseline);

/* detail::cholesky_solve (solver.hpp:98-143) on a row-major PxP matrix; 1 = ok. */
int bfo_cholesky_solve_f32(unsigned p, float *matrix, float *rhs, int scaled);
int bfo_cholesky_solve_f64(unsigned p, double *matrix, double *rhs, int scaled);

/* numerics::add (include/batchfit/numerics.hpp:12-18). */
void bfo_kahan_add_f32(float term, float *sum, float *correction);

/* Model eval / analytic Jacobian (include/batchfit/models.hpp:78-185). */
float bfo_eval_f32(int model, float x, const float *params);
double bfo_eval_f64(int model, double x, const double *params);
void bfo_jacobian_f32(int model, float x, const float *params, float *out);
void bfo_jacobian_f64(int model, double x, const double *params, double *out);

/* estimate_uncertainty<T,Model> (include/batchfit/cpu/uncertainty.hpp:12-110) for one
 * fit with the given accepted state. */
int bfo_uncertainty_f32(int model, size_t m, const float *x, const float *params,
                        int32_t fit_status, float chi2, const float *lower, const float *upper,
                        float *covariance, float *stderr_out, int32_t *ustatus);
int bfo_uncertainty_f64(int model, size_t m, const double *x, const double *params,
                        int32_t fit_status, double chi2, const double *lower,
                        const double *upper, double *covariance, double *stderr_out,
                        int32_t *ustatus);

#ifdef __cplusplus
}
#endif
#endif
