// bf_cuda_fit_noalloc: the fit path for callers that must not allocate GPU memory.
//
// Some callers cannot call cudaMalloc: a host whose memory pool already owns the
// whole device, a real-time pipeline that reserves every buffer up front and
// forbids allocation while it runs, or a library callback that may only enqueue
// work on a stream it was handed.  For them this entry point takes device
// pointers for every input and output, runs on the caller's stream, and keeps
// the only scratch the kernels need -- the LM work counter and the data-only
// guesses -- in a fixed array of static device memory in this file.
//
// The array is kNoAllocScratchBytes (4 MiB).  Every GPU that loads the library
// holds it until the process exits.  All calls share it and it keeps the last
// call's contents; the counter is cleared at the start of every call, and calls
// whose work overlaps on the GPU race on it.
#include "batchfit_cuda.h"
#include "bf_kernels.h"

#include <string>

namespace bf {
namespace host {
int prepare(const bf_fit_args *args, const bf_fit_outputs *out, FitArgs *base, int *lanes);
int report(int code, const std::string &message);
int report_cuda(cudaError_t e, const char *what);
} // namespace host
} // namespace bf

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;
constexpr size_t kCounterBytes = 256; // the work counter, padded to the guess buffer's alignment

// Layout: [0, 8) LM work counter; [256, end) guesses[N*P] when p0 is NULL.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The device address of the scratch array in the calling thread's current CUDA
// context.  In host code the array's name is only a stand-in, not a device
// address.  The address belongs to a context, not to a device (a caller may run
// in a context of its own, or after cudaDeviceReset), so it is looked up on every
// call; the lookup reads the runtime's module table and allocates nothing.  The
// first lookup in a context loads this file's module, which places the array.
int scratch_in_current_context(unsigned char **out) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
        return bf::host::report_cuda(e, "cudaGetSymbolAddress(no-allocation scratch)");
    *out = static_cast<unsigned char *>(ptr);
    return BF_OK;
}

int parameters(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }

// Fits whose guesses fit the scratch: 349,504 (P=3), 262,128 (P=4), 131,064 (P=8).
uint64_t max_guessed_fits(int model) {
    return (kNoAllocScratchBytes - kCounterBytes) / (sizeof(float) * parameters(model));
}

} // namespace

extern "C" {

int bf_cuda_fit_noalloc(const bf_fit_args *args, const bf_fit_outputs *out, void *stream) {
    bf::FitArgs base{};
    int lanes = 0;
    int rc = bf::host::prepare(args, out, &base, &lanes);
    if (rc != BF_OK)
        return rc;
    if (args->memory != BF_MEMORY_DEVICE)
        return bf::host::report(BF_ERR_INVALID_ARGUMENT, "bf_cuda_fit_noalloc takes device memory only");
    if (args->y_format != BF_Y_FLOAT32)
        return bf::host::report(BF_ERR_INVALID_ARGUMENT, "bf_cuda_fit_noalloc takes float32 y (BF_Y_FLOAT32)");
    if (!args->p0 && args->n > max_guessed_fits(args->model))
        return bf::host::report(
            BF_ERR_INVALID_ARGUMENT,
            "bf_cuda_fit_noalloc: N=" + std::to_string(args->n) + " fits without p0 exceed the " +
                std::to_string(max_guessed_fits(args->model)) +
                " whose guesses fit the 4 MiB no-allocation scratch; pass p0 or split the batch");
    if (!args->p0 && args->m > uint32_t(bf::long_guess_smem_max_points()))
        return bf::host::report(
            BF_ERR_INVALID_ARGUMENT,
            "bf_cuda_fit_noalloc: data-only guesses of M=" + std::to_string(args->m) +
                " points need scratch beyond shared memory (M up to " +
                std::to_string(bf::long_guess_smem_max_points()) + " without p0); pass p0");
    unsigned char *scratch = nullptr;
    rc = scratch_in_current_context(&scratch);
    if (rc != BF_OK)
        return rc;
    int device = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
        return bf::host::report_cuda(e, "device attributes");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto *counter = reinterpret_cast<unsigned long long *>(scratch);
    float *guesses = reinterpret_cast<float *>(scratch + kCounterBytes);
    const float *p0 = args->p0;
    if (args->n == 0) {
        // A warm-up: the scratch is placed and the kernels of (model, M, lanes) are
        // loaded on this device; nothing is launched.
        bf::FitArgs a = base;
        a.n = 0;
        e = bf::launch_guess(args->model, nullptr, nullptr, 0, int(args->m), nullptr, nullptr, sms, st);
        if (e == cudaSuccess)
            e = bf::launch_fit(args->model, lanes, a, sms, st, nullptr);
        return e == cudaSuccess ? BF_OK : bf::host::report_cuda(e, "loading the fit kernels");
    }
    if (!p0) {
        e = bf::launch_guess(args->model, args->x, args->y, (long long)args->n, int(args->m), guesses,
                             nullptr, sms, st);
        if (e != cudaSuccess)
            return bf::host::report_cuda(e, "guess kernel");
        p0 = guesses;
    }
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return bf::host::report_cuda(e, "clearing the work counter");
    bf::FitArgs a = base;
    a.x = args->x;
    a.y = args->y;
    a.p0 = p0;
    a.params = out->params;
    a.status = out->status;
    a.iterations = out->iterations;
    a.chi2 = out->chi2;
    a.covariance = out->covariance;
    a.stderr_out = out->standard_errors;
    a.ustatus = out->uncertainty_status;
    a.n = (long long)args->n;
    a.work_counter = counter;
    e = bf::launch_fit(args->model, lanes, a, sms, st, nullptr);
    if (e != cudaSuccess)
        return bf::host::report_cuda(e, "LM kernel");
    return BF_OK;
}

} // extern "C"
