// Kernel argument blocks shared by the host runtime and the device code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bf {

enum : uint32_t { kFlagCompensated = 1u, kFlagScaledCholesky = 2u };
enum : uint32_t { kPolicyReference = 0u, kPolicyParity = 1u };

// Kernel arguments (by value).  Pointers are device pointers.
struct FitArgs {
    const float *x, *y, *p0; // p0 == nullptr: data-only guesses
    float *params, *chi2, *covariance, *stderr_out;
    int32_t *status, *ustatus;
    uint32_t *iterations;
    unsigned long long *work_counter; // dynamic fit claiming; nullptr = static stride
    long long n;
    int m;
    int uncertainties;
    int y_half; // y holds IEEE binary16 values (staged to float32)
    uint32_t max_iterations;
    uint32_t flags;    // kFlagScaledCholesky honoured; sums are always compensated
    uint32_t policy;   // kPolicyReference or kPolicyParity
    uint32_t options_ok; // host-validated lambda/tolerances/bounds (solver.hpp:208-222)
    double lambda0, gtol, xtol, ftol;
    double noise_floor, step_quantum; // parity policy multipliers of FLT_EPSILON
    float lower[8], upper[8];
};

// Values derived from a shared x grid (computed once per CTA, or once per batch
// segment).
struct XConst {
    int m;
    int x_finite;        // every x finite (solver.hpp:223-226)
    int varied_x;        // some x differs from x[0] (solver.hpp:238-239)
    float spacing;       // detail::grid_spacing (solver.hpp:58-69)
    int guess_ok;        // M>=5, finite, strictly increasing, finite span (initial_guess.hpp:131-141)
    float guess_spacing; // min x[j]-x[j-1] (initial_guess.hpp:133-139)
    int count;           // max(1, M/10) edge samples per side (initial_guess.hpp:142)
    int n1;              // power of two >= count (sorting width per side)
    float left_x, right_x; // edge-median abscissae (initial_guess.hpp:151-153)
};

struct LaunchInfo {
    int grid, block, smem, blocks_per_sm, group_lanes;
};

// Measured pipe throughputs (roofline denominators).
struct PeakRates {
    double fp32_tflops, fp64_tflops, mufu_ex2_gops, mufu_rcp_gops;
};

} // namespace bf
