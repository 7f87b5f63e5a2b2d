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
    uint32_t max_iterations;
    uint32_t flags;    // kFlagScaledCholesky honoured; sums are always compensated
    uint32_t policy;   // kPolicyReference or kPolicyParity
    uint32_t options_ok; // host-validated lambda/tolerances/bounds (solver.hpp:208-222)
    double lambda0, gtol, xtol, ftol;
    double noise_floor, step_quantum; // parity policy multipliers of FLT_EPSILON
    float lower[8], upper[8];
};

struct LaunchInfo {
    int grid, block, smem, blocks_per_sm, group_lanes;
};

// Measured pipe throughputs (roofline denominators).
struct PeakRates {
    double fp32_tflops, fp64_tflops, mufu_ex2_gops, mufu_rcp_gops;
};

} // namespace bf
