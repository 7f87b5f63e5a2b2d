// Host-side state of a bf_cuda_context, shared by the C ABI translation units.
#pragma once

#include "batchfit_cuda.h"
#include "bf_args.h"

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace bf {
namespace host {

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t need) {
        if (need <= bytes)
            return cudaSuccess;
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        const cudaError_t e = cudaMalloc(&ptr, need);
        if (e == cudaSuccess)
            bytes = need;
        return e;
    }
    void release() {
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Device-side storage of one in-flight chunk.
struct Slot {
    DeviceBuffer y, p0, guess, params, status, iterations, chi2, cov, se, ustatus, counter;
    DeviceBuffer scratch; // long-spectrum guess scratch when it exceeds shared memory
};

constexpr int kSlots = 2;

struct BatchState; // mixed-batch arena and graph (bf_batch.cu)
void release_batch_state(BatchState *state);

// Shared by the C ABI translation units (bf_capi.cu).
int prepare(const bf_fit_args *args, const bf_fit_outputs *out, FitArgs *base, int *lanes);
// Checks of one mixed-batch segment (M up to max_points) and its kernel arguments.
int prepare_segment(const bf_fit_args *args, const bf_fit_outputs *out, uint32_t max_points, FitArgs *base);
// Group width the single-batch path picks for (model, M).
int default_lanes(int model, uint32_t m);
// Whether a fit call in device memory runs on the single-call group kernels
// (float32 y, the group layout's M; a guess needs the shared-memory guess).
bool single_call_kernels_fit(const bf_fit_args &dev_args);
// Enqueue a validated fit call in device memory on `st` with the single-call
// kernels (guess, LM, covariance), as bf_cuda_fit runs it: `guesses` holds N*P
// floats when p0 is null, `counter` one work counter; grids for `sms` SMs' blocks.
// Nothing is synchronised or timed.
int launch_single_call(const bf_fit_args &dev_args, const bf_fit_outputs &dev_out, float *guesses,
                       unsigned long long *counter, int sms, cudaStream_t st);
int report(int code, const std::string &message);
int report_cuda(cudaError_t e, const char *what);
// Mixed batches (bf_batch.cu): plan, upload and run synchronously on stream[0].
int run_batch(bf_cuda_context *ctx, const bf_batch_segment *segments, uint32_t count, uint32_t flags);
int batch_state(bf_cuda_context *ctx, BatchState **out);
bf_tuning &tuning_of(BatchState *st);
// A batch arena of its own (the server keeps two, one per stream).
int create_batch_state(BatchState **out);
int launch_planned(BatchState &st, const bf_batch_segment *segments, uint32_t count, uint32_t flags, int sms,
                   cudaStream_t stream, bool *launched, bool *graph_used);
int finish_planned(BatchState &st, bool graph_used, bf_cuda_timing *out);
int prepare_planned(BatchState &st, size_t segs, size_t fits, int sms, cudaStream_t stream);
// True once the batch launched on `st` has completed (cudaEventQuery), false while
// it runs; CUDA errors are returned through *error.
bool planned_done(BatchState &st, cudaError_t *error);

// Events around the kernels of one batch: guess = [start, guessed), LM =
// [guessed, fitted), covariance = [fitted, done).
struct KernelEvents {
    cudaEvent_t start, guessed, fitted, done;
};

} // namespace host
} // namespace bf

struct bf_cuda_context {
    int device = 0;
    int sms = 0;
    std::mutex mutex;
    std::atomic<bool> busy{false};
    cudaStream_t stream[bf::host::kSlots] = {nullptr, nullptr};
    cudaEvent_t start = nullptr, stop = nullptr, joined = nullptr;
    bf::host::DeviceBuffer x;
    bf::host::Slot slot[bf::host::kSlots];
    bf_cuda_timing last{};
    // Kernel events of the in-flight submission (one set per chunk).
    std::vector<bf::host::KernelEvents> kernel_events;
    std::vector<cudaEvent_t> event_pool;
    int launches = 0;
    int lanes = 0;
    bf::LaunchInfo info{};
    bf::host::BatchState *batch = nullptr; // created by the first mixed batch
};

