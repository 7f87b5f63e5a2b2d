// Host runtime and C ABI of the batchfit B200 backend (include/batchfit_cuda.h).
//
// A context owns one device, two streams, reusable device staging buffers and the
// per-stream work counters of the persistent kernels.  Device-memory calls launch
// one kernel over all fits.  Host-memory calls run a chunked pipeline: chunk c is
// copied in, fitted and copied out on stream c % 2, so the copies of one chunk
// overlap the kernel of the other.
#include "batchfit_cuda.h"
#include "bf_context.h"
#include "bf_kernels.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

using bf::host::DeviceBuffer;
using bf::host::KernelEvents;
using bf::host::kSlots;
using bf::host::Slot;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &message) {
    g_last_error = message;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(BF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BF_CUDA(call)                                                                              \
    do {                                                                                           \
        const cudaError_t bf_e = (call);                                                           \
        if (bf_e != cudaSuccess)                                                                   \
            return cuda_fail(bf_e, #call);                                                         \
    } while (0)

int parameter_count(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }

// Guess-only outputs (bf_cuda_guess); null members in a fit.
struct GuessOnly {
    float *params;
    int32_t *status;
};


} // namespace

struct bf_cuda_pending {
    bf_cuda_context *ctx;
    int result;
};

namespace {

constexpr int kSmemLimit = 227 * 1024;

// Lanes per fit of the group kernels (8, 16 or 32) for (model, M).
int choose_group_lanes(int model, uint32_t m, int requested) {
    int lanes = requested;
    if (lanes != 8 && lanes != 16 && lanes != 32) {
        // Points per lane between ~8 and ~128 keeps the group reduction and the FP64
        // control amortised without starving the scheduler of independent fits.  The
        // two-Lorentzian pass carries 8 parameters and 36 J^T J sums per point, so its
        // groups widen sooner.  Measured on B200 (LM kernel, ~64M points per call):
        // two-Lorentzian 16 lanes fastest from M=256 to 2048 (M=1024: 3.85 ms vs 5.19
        // at 8, 4.76 at 32), 32 at 4096; the other models 8 lanes up to M=768, 16 at
        // M=1024 (Lorentzian 0.364 vs 0.387 ms at 8) and 1536, 32 from M=2048
        // (pseudo-Voigt 0.506 vs 0.513 at 16).
        if (model == 3)
            lanes = m <= 128 ? 8 : m <= 2048 ? 16 : 32;
        else
            lanes = m < 1024 ? 8 : m < 2048 ? 16 : 32;
    }
    // Fewer, wider groups per CTA when the per-group spectrum buffers do not fit.
    while (lanes < 32 && bf::group_smem_bytes(model, lanes, int(m)) > kSmemLimit)
        lanes *= 2;
    return lanes;
}

// From this M on, the automatic choice is one CTA per fit.  Measured on B200 (LM
// kernel, ~64M points per call): at M = 4096 the 32-lane groups are faster
// (pseudo-Voigt 0.52 vs 0.65 ms, two-Lorentzian 3.40 vs 4.17, Lorentzian 0.35 vs
// 0.44), at M = 8192 one CTA per fit is (0.53 vs 0.68, 2.65 vs 3.01, 0.34 vs 0.46).
constexpr uint32_t kCtaMinPoints = 6144;

// Lanes per fit of a bf_cuda_fit call: a group width, or bf::kCtaLanes (one CTA per
// fit) when asked for, for long spectra, or when the spectrum does not fit the group
// layout.
int choose_lanes(int model, uint32_t m, int requested) {
    if (requested == bf::kCtaLanes || (requested == 0 && m >= kCtaMinPoints))
        return bf::kCtaLanes;
    const int lanes = choose_group_lanes(model, m, requested);
    return bf::group_smem_bytes(model, lanes, int(m)) > kSmemLimit ? bf::kCtaLanes : lanes;
}

bool options_valid(const bf_solver_options &o, int p) {
    if (!std::isfinite(o.initial_lambda) || o.initial_lambda <= 0.0)
        return false;
    for (double t : {o.gradient_tolerance, o.step_tolerance, o.cost_tolerance})
        if (!std::isfinite(t) || t < 0.0)
            return false;
    for (int k = 0; k < p; ++k) {
        const float lo = o.lower[k], hi = o.upper[k];
        if (std::isnan(lo) || std::isnan(hi) || lo > hi || lo == std::numeric_limits<float>::infinity() ||
            hi == -std::numeric_limits<float>::infinity())
            return false;
    }
    return true;
}

bf::FitArgs make_args(const bf_fit_args &in, int p) {
    bf::FitArgs a{};
    const bf_solver_options &o = in.options;
    a.m = int(in.m);
    a.uncertainties = in.uncertainties ? 1 : 0;
    a.y_half = in.y_format == BF_Y_FLOAT16 ? 1 : 0;
    a.max_iterations = o.max_iterations;
    a.flags = (o.compensated_sum ? bf::kFlagCompensated : 0u) | (o.scaled_cholesky ? bf::kFlagScaledCholesky : 0u);
    a.policy = o.policy == BF_POLICY_PARITY ? bf::kPolicyParity : bf::kPolicyReference;
    a.options_ok = options_valid(o, p) ? 1u : 0u;
    if (a.policy == bf::kPolicyReference) {
        // The reference float solver holds lambda and tolerances as float.
        a.lambda0 = double(float(o.initial_lambda));
        a.gtol = double(float(o.gradient_tolerance));
        a.xtol = double(float(o.step_tolerance));
        a.ftol = double(float(o.cost_tolerance));
    } else {
        a.lambda0 = o.initial_lambda;
        a.gtol = o.gradient_tolerance;
        a.xtol = o.step_tolerance;
        a.ftol = o.cost_tolerance;
    }
    a.noise_floor = o.noise_floor;
    a.step_quantum = o.step_quantum;
    for (int k = 0; k < 8; ++k) {
        a.lower[k] = k < p ? o.lower[k] : -std::numeric_limits<float>::infinity();
        a.upper[k] = k < p ? o.upper[k] : std::numeric_limits<float>::infinity();
    }
    return a;
}

// limit == 0: the largest M of the shared-memory kernels for the model.
int validate(const bf_fit_args *args, const bf_fit_outputs *out, uint32_t limit = 0) {
    if (!args || !out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null argument block");
    if (args->model < 0 || args->model > 3)
        return fail(BF_ERR_INVALID_ARGUMENT, "unknown model id");
    if (args->m == 0)
        return fail(BF_ERR_INVALID_ARGUMENT, "fit requires nonempty x[M] (M > 0)");
    if (args->memory != BF_MEMORY_HOST && args->memory != BF_MEMORY_DEVICE)
        return fail(BF_ERR_INVALID_ARGUMENT, "memory must be BF_MEMORY_HOST or BF_MEMORY_DEVICE");
    if (limit == 0)
        limit = uint32_t(bf::kMaxPoints);
    if (args->m > limit)
        return fail(BF_ERR_INVALID_ARGUMENT,
                    "M=" + std::to_string(args->m) + " exceeds this backend's limit of " + std::to_string(limit));
    const int p = parameter_count(args->model);
    if (args->n > uint64_t(std::numeric_limits<int64_t>::max()) / (uint64_t(args->m) + uint64_t(p) * p))
        return fail(BF_ERR_INVALID_ARGUMENT, "N*M or N*P*P overflows 64-bit indexing");
    if (args->group_lanes != 0 && args->group_lanes != 8 && args->group_lanes != 16 && args->group_lanes != 32 &&
        args->group_lanes != bf::kCtaLanes)
        return fail(BF_ERR_INVALID_ARGUMENT, "group_lanes must be 0, 8, 16, 32 or 128 (one CTA per fit)");
    if (args->y_format != BF_Y_FLOAT32 && args->y_format != BF_Y_FLOAT16)
        return fail(BF_ERR_INVALID_ARGUMENT, "y_format must be BF_Y_FLOAT32 or BF_Y_FLOAT16");
    if (args->y_format == BF_Y_FLOAT16 &&
        (choose_lanes(args->model, args->m, args->group_lanes) == bf::kCtaLanes ||
         (!args->p0 && args->m > uint32_t(bf::group_guess_max_points()))))
        return fail(BF_ERR_INVALID_ARGUMENT,
                    "half-precision y (BF_Y_FLOAT16) is staged by the group kernels only: M=" +
                        std::to_string(args->m) + " needs float32 y");
    if (args->n == 0)
        return BF_OK;
    if (!args->x || !args->y)
        return fail(BF_ERR_INVALID_ARGUMENT, "x and y are required");
    if (!out->params || !out->status || !out->iterations || !out->chi2)
        return fail(BF_ERR_INVALID_ARGUMENT, "params, status, iterations and chi2 outputs are required");
    if (args->uncertainties && (!out->covariance || !out->standard_errors || !out->uncertainty_status))
        return fail(BF_ERR_INVALID_ARGUMENT, "uncertainty outputs are required when uncertainties is set");
    return BF_OK;
}

cudaEvent_t take_event(bf_cuda_context *ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Launch the kernels of one batch already resident on the device: the data-only
// guess when there are no initial values (into `guess_buf`), then the LM kernel.
int launch_batch(bf_cuda_context *ctx, const bf_fit_args &in, const bf::FitArgs &base, int lanes, const float *x,
                 const float *y, const float *p0, float *guess_buf, int32_t *guess_status, bool guess_only,
                 const bf_fit_outputs &dev_out, unsigned long long *counter, long long count, cudaStream_t st,
                 bf::host::DeviceBuffer &scratch) {
    // Four events bracket the guess, LM and covariance kernels of this batch.
    KernelEvents ev{take_event(ctx), take_event(ctx), take_event(ctx), take_event(ctx)};
    BF_CUDA(cudaEventRecord(ev.start, st));
    if (!p0 || guess_only) {
        const size_t scratch_bytes =
            in.m > uint32_t(bf::group_guess_max_points()) ? bf::long_guess_scratch_bytes(int(in.m), ctx->sms) : 0;
        if (scratch_bytes)
            BF_CUDA(scratch.reserve(scratch_bytes));
        BF_CUDA(bf::launch_guess(in.model, x, y, count, int(in.m), guess_buf, guess_status, ctx->sms, st,
                                 base.y_half, scratch_bytes ? static_cast<float *>(scratch.ptr) : nullptr));
        ++ctx->launches;
        p0 = guess_buf;
    }
    BF_CUDA(cudaEventRecord(ev.guessed, st));
    if (!guess_only) {
        bf::FitArgs a = base;
        a.x = x;
        a.y = y;
        a.p0 = p0;
        a.params = dev_out.params;
        a.status = dev_out.status;
        a.iterations = dev_out.iterations;
        a.chi2 = dev_out.chi2;
        a.covariance = dev_out.covariance;
        a.stderr_out = dev_out.standard_errors;
        a.ustatus = dev_out.uncertainty_status;
        a.n = count;
        a.work_counter = counter;
        BF_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
        BF_CUDA(bf::launch_fit(in.model, lanes, a, ctx->sms, st, &ctx->info, ev.fitted));
        ctx->launches += in.uncertainties ? 2 : 1; // LM kernel (+ covariance kernel)
    } else {
        BF_CUDA(cudaEventRecord(ev.fitted, st));
    }
    BF_CUDA(cudaEventRecord(ev.done, st));
    ctx->kernel_events.push_back(ev);
    return BF_OK;
}

// Enqueue a whole fit (or guess-only run) on the context's streams.
int enqueue(bf_cuda_context *ctx, const bf_fit_args &in, const bf_fit_outputs &out, const GuessOnly *guess_only) {
    const int p = parameter_count(in.model);
    const uint64_t n = in.n, m = in.m;
    const int lanes = choose_lanes(in.model, in.m, in.group_lanes);
    ctx->lanes = lanes;
    ctx->launches = 0;
    ctx->info = bf::LaunchInfo{};
    for (auto &ev : ctx->kernel_events)
        for (cudaEvent_t e : {ev.start, ev.guessed, ev.fitted, ev.done})
            ctx->event_pool.push_back(e);
    ctx->kernel_events.clear();
    BF_CUDA(cudaSetDevice(ctx->device));
    BF_CUDA(cudaEventRecord(ctx->start, ctx->stream[0]));
    BF_CUDA(cudaStreamWaitEvent(ctx->stream[1], ctx->start, 0));
    const bf::FitArgs base = make_args(in, p);
    const bool need_guess = in.p0 == nullptr || guess_only != nullptr;

    if (in.memory == BF_MEMORY_DEVICE) {
        Slot &s = ctx->slot[0];
        BF_CUDA(s.counter.reserve(sizeof(unsigned long long)));
        float *gbuf = nullptr;
        int32_t *gstat = nullptr;
        if (guess_only) {
            gbuf = guess_only->params;
            gstat = guess_only->status;
        } else if (need_guess) {
            BF_CUDA(s.guess.reserve(n * p * sizeof(float)));
            gbuf = static_cast<float *>(s.guess.ptr);
        }
        if (n > 0) {
            const int rc = launch_batch(ctx, in, base, lanes, in.x, in.y, in.p0, gbuf, gstat, guess_only != nullptr,
                                        out, static_cast<unsigned long long *>(s.counter.ptr), (long long)n,
                                        ctx->stream[0], s.scratch);
            if (rc != BF_OK)
                return rc;
        }
        BF_CUDA(cudaEventRecord(ctx->stop, ctx->stream[0]));
        return BF_OK;
    }
    if (guess_only)
        return fail(BF_ERR_INVALID_ARGUMENT, "guess-only runs take device memory");

    // Host memory: x once, then double-buffered chunks.
    BF_CUDA(ctx->x.reserve(m * sizeof(float)));
    BF_CUDA(cudaMemcpyAsync(ctx->x.ptr, in.x, m * sizeof(float), cudaMemcpyHostToDevice, ctx->stream[0]));
    cudaEvent_t x_ready = take_event(ctx);
    BF_CUDA(cudaEventRecord(x_ready, ctx->stream[0]));
    BF_CUDA(cudaStreamWaitEvent(ctx->stream[1], x_ready, 0));
    ctx->event_pool.push_back(x_ready);
    // ~128 MB of observations per chunk, at least a few waves of fits.
    const size_t ybytes = in.y_format == BF_Y_FLOAT16 ? 2 : sizeof(float); // bytes per y value
    uint64_t chunk = std::max<uint64_t>(16384, (128ull << 20) / (m * ybytes));
    if (chunk > n)
        chunk = n;
    const bool has_p0 = in.p0 != nullptr;
    for (int i = 0; i < kSlots && n > 0; ++i) {
        Slot &s = ctx->slot[i];
        BF_CUDA(s.y.reserve(chunk * m * ybytes));
        if (has_p0)
            BF_CUDA(s.p0.reserve(chunk * p * sizeof(float)));
        else
            BF_CUDA(s.guess.reserve(chunk * p * sizeof(float)));
        BF_CUDA(s.params.reserve(chunk * p * sizeof(float)));
        BF_CUDA(s.status.reserve(chunk * sizeof(int32_t)));
        BF_CUDA(s.iterations.reserve(chunk * sizeof(uint32_t)));
        BF_CUDA(s.chi2.reserve(chunk * sizeof(float)));
        if (in.uncertainties) {
            BF_CUDA(s.cov.reserve(chunk * p * p * sizeof(float)));
            BF_CUDA(s.se.reserve(chunk * p * sizeof(float)));
            BF_CUDA(s.ustatus.reserve(chunk * sizeof(int32_t)));
        }
        BF_CUDA(s.counter.reserve(sizeof(unsigned long long)));
    }
    int c = 0;
    for (uint64_t first = 0; first < n; first += chunk, ++c) {
        const uint64_t count = std::min(chunk, n - first);
        Slot &s = ctx->slot[c % kSlots];
        cudaStream_t st = ctx->stream[c % kSlots];
        BF_CUDA(cudaMemcpyAsync(s.y.ptr, reinterpret_cast<const char *>(in.y) + first * m * ybytes,
                                count * m * ybytes, cudaMemcpyHostToDevice, st));
        if (has_p0)
            BF_CUDA(cudaMemcpyAsync(s.p0.ptr, in.p0 + first * p, count * p * sizeof(float), cudaMemcpyHostToDevice,
                                    st));
        const bf_fit_outputs dev_out{static_cast<float *>(s.params.ptr),     static_cast<int32_t *>(s.status.ptr),
                                     static_cast<uint32_t *>(s.iterations.ptr), static_cast<float *>(s.chi2.ptr),
                                     static_cast<float *>(s.cov.ptr),        static_cast<float *>(s.se.ptr),
                                     static_cast<int32_t *>(s.ustatus.ptr)};
        const int rc = launch_batch(ctx, in, base, lanes, static_cast<const float *>(ctx->x.ptr),
                                    static_cast<const float *>(s.y.ptr),
                                    has_p0 ? static_cast<const float *>(s.p0.ptr) : nullptr,
                                    static_cast<float *>(s.guess.ptr), nullptr, false, dev_out,
                                    static_cast<unsigned long long *>(s.counter.ptr), (long long)count, st,
                                    s.scratch);
        if (rc != BF_OK)
            return rc;
        auto d2h = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
        };
        BF_CUDA(d2h(out.params + first * p, s.params.ptr, count * p * sizeof(float)));
        BF_CUDA(d2h(out.status + first, s.status.ptr, count * sizeof(int32_t)));
        BF_CUDA(d2h(out.iterations + first, s.iterations.ptr, count * sizeof(uint32_t)));
        BF_CUDA(d2h(out.chi2 + first, s.chi2.ptr, count * sizeof(float)));
        if (in.uncertainties) {
            BF_CUDA(d2h(out.covariance + first * p * p, s.cov.ptr, count * p * p * sizeof(float)));
            BF_CUDA(d2h(out.standard_errors + first * p, s.se.ptr, count * p * sizeof(float)));
            BF_CUDA(d2h(out.uncertainty_status + first, s.ustatus.ptr, count * sizeof(int32_t)));
        }
    }
    BF_CUDA(cudaEventRecord(ctx->joined, ctx->stream[1]));
    BF_CUDA(cudaStreamWaitEvent(ctx->stream[0], ctx->joined, 0));
    BF_CUDA(cudaEventRecord(ctx->stop, ctx->stream[0]));
    return BF_OK;
}

int finish(bf_cuda_context *ctx) {
    BF_CUDA(cudaEventSynchronize(ctx->stop));
    float total = 0.0f;
    BF_CUDA(cudaEventElapsedTime(&total, ctx->start, ctx->stop));
    double kernel = 0.0, guess = 0.0, lm = 0.0, cov = 0.0;
    for (auto &ev : ctx->kernel_events) {
        float t[3] = {0.0f, 0.0f, 0.0f};
        BF_CUDA(cudaEventElapsedTime(&t[0], ev.start, ev.guessed));
        BF_CUDA(cudaEventElapsedTime(&t[1], ev.guessed, ev.fitted));
        BF_CUDA(cudaEventElapsedTime(&t[2], ev.fitted, ev.done));
        guess += t[0];
        lm += t[1];
        cov += t[2];
        kernel += double(t[0]) + t[1] + t[2];
    }
    ctx->last.kernel_ms = kernel;
    ctx->last.guess_ms = guess;
    ctx->last.lm_ms = lm;
    ctx->last.covariance_ms = cov;
    ctx->last.batches = uint32_t(ctx->kernel_events.size());
    ctx->last.total_ms = total;
    ctx->last.launches = uint32_t(ctx->launches);
    ctx->last.group_lanes = ctx->lanes;
    ctx->last.grid = ctx->info.grid;
    ctx->last.blocks_per_sm = ctx->info.blocks_per_sm;
    return BF_OK;
}

} // namespace

// Shared with bf_noalloc.cu: argument checks, kernel arguments and the group width
// of a device-memory fit, and the thread-local error report.
namespace bf {
namespace host {
int prepare(const bf_fit_args *args, const bf_fit_outputs *out, FitArgs *base, int *lanes) {
    const int rc = validate(args, out);
    if (rc != BF_OK)
        return rc;
    *base = make_args(*args, parameter_count(args->model));
    *lanes = choose_lanes(args->model, args->m, args->group_lanes);
    return BF_OK;
}
int prepare_segment(const bf_fit_args *args, const bf_fit_outputs *out, uint32_t max_points, FitArgs *base) {
    const int rc = validate(args, out, max_points);
    if (rc != BF_OK)
        return rc;
    if (args->y_format != BF_Y_FLOAT32)
        return fail(BF_ERR_INVALID_ARGUMENT, "this entry point takes float32 y (BF_Y_FLOAT32)");
    *base = make_args(*args, parameter_count(args->model));
    return BF_OK;
}
int default_lanes(int model, uint32_t m) { return choose_group_lanes(model, m, 0); }
bool single_call_kernels_fit(const bf_fit_args &a) {
    if (a.y_format != BF_Y_FLOAT32 || choose_lanes(a.model, a.m, a.group_lanes) == bf::kCtaLanes)
        return false;
    return a.p0 || a.m <= uint32_t(bf::group_guess_max_points());
}
int launch_single_call(const bf_fit_args &a, const bf_fit_outputs &out, float *guesses, unsigned long long *counter,
                       int sms, cudaStream_t st) {
    const int p = parameter_count(a.model);
    const int lanes = choose_lanes(a.model, a.m, a.group_lanes);
    bf::FitArgs f = make_args(a, p);
    const long long n = (long long)a.n;
    const float *p0 = a.p0;
    if (!p0) {
        BF_CUDA(bf::launch_guess(a.model, a.x, a.y, n, int(a.m), guesses, nullptr, sms, st, 0, nullptr));
        p0 = guesses;
    }
    f.x = a.x;
    f.y = a.y;
    f.p0 = p0;
    f.params = out.params;
    f.status = out.status;
    f.iterations = out.iterations;
    f.chi2 = out.chi2;
    f.covariance = out.covariance;
    f.stderr_out = out.standard_errors;
    f.ustatus = out.uncertainty_status;
    f.n = n;
    f.work_counter = counter;
    BF_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
    bf::LaunchInfo info{};
    BF_CUDA(bf::launch_fit(a.model, lanes, f, sms, st, &info, nullptr));
    return BF_OK;
}
int report(int code, const std::string &message) { return fail(code, message); }
int report_cuda(cudaError_t e, const char *what) { return cuda_fail(e, what); }
} // namespace host
} // namespace bf

extern "C" {

const char *bf_cuda_last_error(void) { return g_last_error.c_str(); }

int bf_cuda_version(void) { return 10; }

int bf_cuda_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop{};
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10)
            return 1;
    }
    return 0;
}

uint32_t bf_cuda_max_points(int32_t model) {
    if (model < 0 || model > 3)
        return 0;
    return uint32_t(bf::kMaxPoints);
}

int bf_cuda_context_create(int device, bf_cuda_context **out) {
    if (!out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(BF_ERR_UNAVAILABLE, "CUDA fitting is unavailable: no CUDA device");
    }
    if (device < 0 || device >= count)
        return fail(BF_ERR_INVALID_ARGUMENT, "device index out of range");
    cudaDeviceProp prop{};
    BF_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(BF_ERR_UNAVAILABLE, std::string("CUDA fitting is unavailable: device '") + prop.name +
                                            "' is not sm_100 (this build targets sm_100a only)");
    auto *ctx = new bf_cuda_context();
    ctx->device = device;
    ctx->sms = prop.multiProcessorCount;
    cudaError_t e = cudaSetDevice(device);
    for (int i = 0; i < kSlots && e == cudaSuccess; ++i)
        e = cudaStreamCreateWithFlags(&ctx->stream[i], cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaEventCreate(&ctx->start);
    if (e == cudaSuccess)
        e = cudaEventCreate(&ctx->stop);
    if (e == cudaSuccess)
        e = cudaEventCreate(&ctx->joined);
    if (e != cudaSuccess) {
        bf_cuda_context_destroy(ctx);
        return cuda_fail(e, "context setup");
    }
    *out = ctx;
    return BF_OK;
}

void bf_cuda_context_destroy(bf_cuda_context *ctx) {
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    for (auto &st : ctx->stream)
        if (st)
            cudaStreamSynchronize(st);
    for (auto &s : ctx->slot) {
        s.y.release();
        s.p0.release();
        s.guess.release();
        s.params.release();
        s.status.release();
        s.iterations.release();
        s.chi2.release();
        s.cov.release();
        s.se.release();
        s.ustatus.release();
        s.counter.release();
        s.scratch.release();
    }
    ctx->x.release();
    bf::host::release_batch_state(ctx->batch);
    ctx->batch = nullptr;
    for (auto &ev : ctx->kernel_events)
        for (cudaEvent_t e : {ev.start, ev.guessed, ev.fitted, ev.done})
            cudaEventDestroy(e);
    for (auto ev : ctx->event_pool)
        cudaEventDestroy(ev);
    for (cudaEvent_t ev : {ctx->start, ctx->stop, ctx->joined})
        if (ev)
            cudaEventDestroy(ev);
    for (auto &st : ctx->stream)
        if (st)
            cudaStreamDestroy(st);
    delete ctx;
}

int bf_cuda_default_options(int32_t model, uint32_t policy, bf_solver_options *out) {
    if (!out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null output pointer");
    if (model < 0 || model > 3)
        return fail(BF_ERR_INVALID_ARGUMENT, "unknown model id");
    if (policy != BF_POLICY_REFERENCE && policy != BF_POLICY_PARITY)
        return fail(BF_ERR_INVALID_ARGUMENT, "unknown policy");
    bf_solver_options o{};
    o.max_iterations = 100;
    o.initial_lambda = 1e-3;
    // Float defaults (solver.hpp:29-31) for the reference policy, double defaults
    // for the parity policy.
    o.gradient_tolerance = policy == BF_POLICY_PARITY ? 1e-10 : 1e-5;
    o.step_tolerance = policy == BF_POLICY_PARITY ? 1e-10 : 1e-6;
    o.cost_tolerance = policy == BF_POLICY_PARITY ? 1e-12 : 1e-6;
    o.compensated_sum = 1;
    o.scaled_cholesky = 0;
    o.policy = policy;
    o.noise_floor = 16.0;
    o.step_quantum = 16.0;
    for (int k = 0; k < 8; ++k) {
        o.lower[k] = -std::numeric_limits<float>::infinity();
        o.upper[k] = std::numeric_limits<float>::infinity();
    }
    *out = o;
    return BF_OK;
}

int bf_cuda_submit(bf_cuda_context *ctx, const bf_fit_args *args, const bf_fit_outputs *out,
                   bf_cuda_pending **pending) {
    if (!ctx || !pending)
        return fail(BF_ERR_INVALID_ARGUMENT, "null context or pending pointer");
    *pending = nullptr;
    int rc = validate(args, out);
    if (rc != BF_OK)
        return rc;
    if (ctx->busy.exchange(true))
        return fail(BF_ERR_BUSY, "a submission is already in flight on this context");
    {
        std::lock_guard<std::mutex> lock(ctx->mutex);
        rc = enqueue(ctx, *args, *out, nullptr);
    }
    if (rc != BF_OK) {
        // Drain whatever was queued before the failure.
        for (auto &st : ctx->stream)
            cudaStreamSynchronize(st);
        ctx->busy.store(false);
        return rc;
    }
    *pending = new bf_cuda_pending{ctx, BF_OK};
    return BF_OK;
}

int bf_cuda_ready(bf_cuda_pending *pending) {
    if (!pending)
        return -BF_ERR_INVALID_ARGUMENT;
    const cudaError_t e = cudaEventQuery(pending->ctx->stop);
    if (e == cudaSuccess)
        return 1;
    if (e == cudaErrorNotReady)
        return 0;
    cuda_fail(e, "cudaEventQuery");
    return -BF_ERR_CUDA;
}

int bf_cuda_wait(bf_cuda_pending *pending) {
    if (!pending)
        return fail(BF_ERR_INVALID_ARGUMENT, "null pending handle");
    bf_cuda_context *ctx = pending->ctx;
    int rc;
    {
        std::lock_guard<std::mutex> lock(ctx->mutex);
        rc = finish(ctx);
        if (rc == BF_OK) {
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess)
                rc = cuda_fail(e, "fit kernel");
        }
    }
    ctx->busy.store(false);
    delete pending;
    return rc;
}

int bf_cuda_fit(bf_cuda_context *ctx, const bf_fit_args *args, const bf_fit_outputs *out) {
    bf_cuda_pending *pending = nullptr;
    const int rc = bf_cuda_submit(ctx, args, out, &pending);
    if (rc != BF_OK)
        return rc;
    return bf_cuda_wait(pending);
}

int bf_cuda_guess(bf_cuda_context *ctx, int32_t model, uint64_t n, uint32_t m, const float *x, const float *y,
                  int32_t memory, float *params, int32_t *guess_status) {
    if (!ctx)
        return fail(BF_ERR_INVALID_ARGUMENT, "null context");
    bf_fit_args args{};
    args.model = model;
    args.n = n;
    args.m = m;
    args.x = x;
    args.y = y;
    args.memory = memory;
    bf_cuda_default_options(model < 0 || model > 3 ? 0 : model, BF_POLICY_REFERENCE, &args.options);
    // The guess-only launch writes no fit outputs; validation needs placeholders.
    float dummy_f = 0.0f;
    int32_t dummy_i = 0;
    uint32_t dummy_u = 0;
    bf_fit_outputs out{&dummy_f, &dummy_i, &dummy_u, &dummy_f, nullptr, nullptr, nullptr};
    int rc = validate(&args, &out);
    if (rc != BF_OK)
        return rc;
    if (n > 0 && (!params || !guess_status))
        return fail(BF_ERR_INVALID_ARGUMENT, "params and guess_status outputs are required");
    if (ctx->busy.exchange(true))
        return fail(BF_ERR_BUSY, "a submission is already in flight on this context");
    std::lock_guard<std::mutex> lock(ctx->mutex);
    const int p = parameter_count(model);
    rc = BF_OK;
    do {
        if (n == 0)
            break;
        if (memory == BF_MEMORY_DEVICE) {
            bf_fit_args a = args;
            const GuessOnly go{params, guess_status};
            rc = enqueue(ctx, a, out, &go);
            if (rc == BF_OK)
                rc = finish(ctx);
            break;
        }
        // Host memory: stage everything on the device once (guesses are cheap).
        DeviceBuffer dx, dy, dp, ds;
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e == cudaSuccess)
            e = dx.reserve(size_t(m) * sizeof(float));
        if (e == cudaSuccess)
            e = dy.reserve(size_t(n) * m * sizeof(float));
        if (e == cudaSuccess)
            e = dp.reserve(size_t(n) * p * sizeof(float));
        if (e == cudaSuccess)
            e = ds.reserve(size_t(n) * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMemcpy(dx.ptr, x, size_t(m) * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(dy.ptr, y, size_t(n) * m * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "guess staging");
        } else {
            bf_fit_args a = args;
            a.x = static_cast<const float *>(dx.ptr);
            a.y = static_cast<const float *>(dy.ptr);
            a.memory = BF_MEMORY_DEVICE;
            const GuessOnly go{static_cast<float *>(dp.ptr), static_cast<int32_t *>(ds.ptr)};
            rc = enqueue(ctx, a, out, &go);
            if (rc == BF_OK)
                rc = finish(ctx);
            if (rc == BF_OK) {
                e = cudaMemcpy(params, dp.ptr, size_t(n) * p * sizeof(float), cudaMemcpyDeviceToHost);
                if (e == cudaSuccess)
                    e = cudaMemcpy(guess_status, ds.ptr, size_t(n) * sizeof(int32_t), cudaMemcpyDeviceToHost);
                if (e != cudaSuccess)
                    rc = cuda_fail(e, "guess readback");
            }
        }
        dx.release();
        dy.release();
        dp.release();
        ds.release();
    } while (false);
    ctx->busy.store(false);
    return rc;
}

int bf_cuda_last_timing(bf_cuda_context *ctx, bf_cuda_timing *out) {
    if (!ctx || !out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null argument");
    *out = ctx->last;
    return BF_OK;
}

int bf_cuda_measure_peaks(bf_cuda_context *ctx, bf_cuda_peaks *out) {
    if (!ctx || !out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null argument");
    if (ctx->busy.exchange(true))
        return fail(BF_ERR_BUSY, "a submission is already in flight on this context");
    std::lock_guard<std::mutex> lock(ctx->mutex);
    bf::PeakRates rates{};
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess)
        e = bf::measure_peaks(ctx->sms, ctx->stream[0], &rates);
    ctx->busy.store(false);
    if (e != cudaSuccess)
        return cuda_fail(e, "peak microbenchmarks");
    out->fp32_tflops = rates.fp32_tflops;
    out->fp64_tflops = rates.fp64_tflops;
    out->mufu_ex2_gops = rates.mufu_ex2_gops;
    out->mufu_rcp_gops = rates.mufu_rcp_gops;
    return BF_OK;
}

int bf_cuda_host_alloc(size_t bytes, void **out) {
    if (!out)
        return fail(BF_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (bytes == 0)
        return BF_OK;
    BF_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
    return BF_OK;
}

int bf_cuda_host_free(void *ptr) {
    if (ptr)
        BF_CUDA(cudaFreeHost(ptr));
    return BF_OK;
}

} // extern "C"
