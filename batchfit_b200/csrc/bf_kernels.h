// Host-side entry points into the fit kernels (implemented in bf_kernels.cu).
#pragma once

#include "bf_args.h"

namespace bf {

// Threads of the CTA-per-fit LM kernel for long spectra (bf_long.cu); also the
// lanes-per-fit value that selects it.
constexpr int kCtaThreads = 128;
constexpr int kCtaLanes = kCtaThreads;
// Largest M of any fit path (int indexing of rows and scratch).
constexpr int kMaxPoints = 1 << 24;

// Launch the persistent LM kernel for `model` with `lanes` (8, 16 or 32) lanes per
// fit on `stream`, followed by the covariance kernel when a.uncertainties.  a.p0
// must hold initial values for every fit (the user's, or the guess kernel's
// output).  The caller zeroes a.work_counter (when non-null) first.  When lm_done
// is non-null it is recorded on `stream` between the two kernels.  With a.n == 0
// nothing is launched: the kernels are only loaded on the current device.
cudaError_t launch_fit(int model, int lanes, const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info,
                       cudaEvent_t lm_done = nullptr);

// lanes == kCtaLanes runs the CTA-per-fit kernel (any M, float32 y).
//
// Launch the data-only guess kernel: guesses[N*P] and, when non-null, status[N].
// Its group width follows from M; y_half: y holds IEEE binary16 values.  With
// n == 0 nothing is launched (x and y may be null): the kernel is only loaded.
// M above group_guess_max_points() runs the long-spectrum guess (float32 y only),
// which needs `gscratch` of long_guess_scratch_bytes(M, sms) bytes when that is
// nonzero.
cudaError_t launch_guess(int model, const float *x, const float *y, long long n, int m, float *guesses,
                         int32_t *status, int sms, cudaStream_t stream, int y_half = 0, float *gscratch = nullptr);

// Dynamic shared memory of one group LM CTA for (model, lanes, M).
int group_smem_bytes(int model, int lanes, int m);
// Largest M of the group LM kernel at 32 lanes per fit (its row must fit shared memory).
int group_lm_max_points(int model);
// Largest M of the group guess kernel.
int group_guess_max_points();

// Long spectra (bf_long.cu).
cudaError_t launch_lm_cta(int model, const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info);
cudaError_t launch_guess_long(int model, const float *x, const float *y, long long n, int m, float *guesses,
                              int32_t *status, int sms, cudaStream_t stream, float *gscratch);
// Global scratch the long guess needs for M (0: its scratch fits shared memory).
size_t long_guess_scratch_bytes(int m, int sms);
// Largest M whose long-guess scratch fits shared memory.
int long_guess_smem_max_points();

// FP32 FMA, FP64 FMA and MUFU ex2/rcp throughput on the current device.
cudaError_t measure_peaks(int sms, cudaStream_t stream, PeakRates *out);

} // namespace bf
