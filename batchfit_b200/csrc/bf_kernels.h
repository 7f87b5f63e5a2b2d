// Host-side entry points into the fit kernels (implemented in bf_kernels.cu).
#pragma once

#include "bf_args.h"

namespace bf {

// Launch the persistent LM kernel for `model` with `lanes` (8, 16 or 32) lanes per
// fit on `stream`, followed by the covariance kernel when a.uncertainties.  a.p0
// must hold initial values for every fit (the user's, or the guess kernel's
// output).  The caller zeroes a.work_counter (when non-null) first.  When lm_done
// is non-null it is recorded on `stream` between the two kernels.  With a.n == 0
// nothing is launched: the kernels are only loaded on the current device.
cudaError_t launch_fit(int model, int lanes, const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info,
                       cudaEvent_t lm_done = nullptr);

// Launch the data-only guess kernel: guesses[N*P] and, when non-null, status[N].
// Its group width follows from M; y_half: y holds IEEE binary16 values.  With
// n == 0 nothing is launched (x and y may be null): the kernel is only loaded.
cudaError_t launch_guess(int model, const float *x, const float *y, long long n, int m, float *guesses,
                         int32_t *status, int sms, cudaStream_t stream, int y_half = 0);

// Dynamic shared memory of one CTA for (model, lanes, M).
int smem_bytes(int model, int lanes, int m);

// Largest M the shared-memory layout supports for `model`.
int max_points(int model);

// FP32 FMA, FP64 FMA and MUFU ex2/rcp throughput on the current device.
cudaError_t measure_peaks(int sms, cudaStream_t stream, PeakRates *out);

} // namespace bf
