// Serving runtime: continuous batching of fit requests on one GPU
// (include/batchfit_cuda.h, "Serving").
//
// One scheduler thread runs the loop
//   intake     new submissions join the pending queue (arrival order);
//   admission  the queue's head is admitted while its device buffers fit the
//              budget: one stream-ordered allocation from the server's memory pool,
//              inputs copied in on the copy stream;
//   launch     when one of the two batch slots is free, the admitted requests whose
//              inputs are on the device (up to max_batch_fits) become one mixed
//              batch on that slot's stream;
//   retire     a slot whose batch finished copies its outputs back, releases the
//              buffers, completes its requests and returns their bytes to the budget.
// With two slots, a batch formed while another runs starts as soon as its inputs
// are on the device and fills the SMs the running batch's tail leaves idle.
#include "batchfit_cuda.h"
#include "bf_batch.h"
#include "bf_context.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using bf::host::report;
using bf::host::report_cuda;
using Clock = std::chrono::steady_clock;

int parameters(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }
size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Completion of one admission round's copies on the copy stream.
struct CopyMark {
    cudaEvent_t event = nullptr;
    ~CopyMark() {
        if (event)
            cudaEventDestroy(event);
    }
};

struct Request {
    uint64_t ticket = 0;
    std::shared_ptr<CopyMark> copied; // its inputs are on the device once this completes
    bf_fit_args args{};         // host pointers of the caller
    bf_fit_outputs host_out{};  // host outputs of the caller
    size_t bytes = 0;           // device bytes charged to the budget
    char *block = nullptr;      // one device allocation for all of the request's buffers
    bf_batch_segment seg{};     // the request with device pointers
    float *guesses = nullptr;   // N*P floats and a work counter: a large request alone
    unsigned long long *counter = nullptr; // runs on the single-call kernels
    Clock::time_point submitted, done;
    int result = BF_OK;
    bool charged = false;   // its bytes count against the budget (admitted)
    bool cancelled = false; // cancelled before admission: completes with BF_ERR_CANCELLED
    bool finished = false;
};

// Predicted device time of a request (ms): N * M points at the per-point cost of
// its model's kernels (guess + LM), measured on B200 at the benchmark sizes.  Only
// ratios matter: the scheduler uses it to keep batches short.
double predicted_ms(const bf_fit_args &a) {
    static constexpr double kNsPerPoint[4] = {0.010, 0.010, 0.014, 0.10};
    return double(a.n) * double(a.m) * kNsPerPoint[a.model & 3] * 1e-6;
}
// A batch grows to about this much predicted device time; a larger request runs alone.
constexpr double kBatchTargetMs = 1.0;

// Device bytes of a request: x, y, p0, outputs, plus the batch arena's per-fit
// share (work items and guesses).
size_t request_bytes(const bf_fit_args &a) {
    const size_t n = a.n, m = a.m, p = size_t(parameters(a.model));
    size_t b = align256(m * 4) + align256(n * m * 4) + (a.p0 ? align256(n * p * 4) : 0);
    b += align256(n * p * 4) + 3 * align256(n * 4) + align256(n * 4); // params, status/iters/chi2, ustatus
    if (a.uncertainties)
        b += align256(n * p * p * 4) + align256(n * p * 4);
    b += n * (2 * sizeof(bf::WorkItem) + p * 4);
    b += align256(n * p * 4) + 256; // guesses and work counter of the single-call kernels
    return b;
}

struct Slot {
    bf::host::BatchState *state = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr; // after the batch, the copies back and the frees
    std::vector<std::shared_ptr<Request>> requests;
    bool busy = false, graph_used = false, launched = false;
    bool large = false; // runs a request predicted to take longer than kBatchTargetMs
};

} // namespace

struct bf_server {
    int device = 0, sms = 0;
    bf_server_options opt{};
    cudaMemPool_t pool = nullptr;
    cudaStream_t copy = nullptr;
    Slot slot[2];
    std::thread worker;
    std::mutex mutex;
    std::condition_variable wake, finished;
    bool stopping = false;
    uint64_t next_ticket = 1;
    std::deque<std::shared_ptr<Request>> incoming;        // submitted, not yet seen by the scheduler
    std::map<uint64_t, std::shared_ptr<Request>> tickets; // every unreleased request
    bf_server_stats stats{};
    std::string fatal; // a CUDA failure that stopped the scheduler
    uint32_t fail_allocations = 0; // host-side fault injection (bf_server_fail_allocations)

    // Scheduler-owned state.
    std::deque<std::shared_ptr<Request>> pending;  // waiting for admission
    std::vector<std::shared_ptr<Request>> ready;   // admitted, copied in, not launched
};

namespace {

void complete(bf_server *s, const std::shared_ptr<Request> &r, int result) {
    std::lock_guard<std::mutex> lock(s->mutex);
    r->result = result;
    r->finished = true;
    r->done = Clock::now();
    if (r->charged)
        s->stats.memory_in_use -= r->bytes;
    r->charged = false;
    s->stats.completed += 1;
    if (result != BF_OK)
        s->stats.failed += 1;
    else
        s->stats.fits_completed += r->args.n;
    s->finished.notify_all();
}

// Admit the head of the queue while it fits: allocate its buffers and queue its
// input copies; the round's copies share one completion mark.  False on a CUDA
// failure.
bool admit(bf_server *s) {
    std::shared_ptr<CopyMark> mark;
    while (!s->pending.empty()) {
        const std::shared_ptr<Request> r = s->pending.front();
        bool cancelled = false, inject = false;
        {
            std::lock_guard<std::mutex> lock(s->mutex);
            cancelled = r->cancelled;
            if (!cancelled) {
                if (s->stats.memory_in_use + r->bytes > s->stats.memory_budget)
                    break;
                s->stats.memory_in_use += r->bytes;
                s->stats.memory_peak = std::max(s->stats.memory_peak, s->stats.memory_in_use);
                r->charged = true;
                if (s->fail_allocations) {
                    s->fail_allocations -= 1;
                    inject = true;
                }
            }
        }
        if (cancelled) {
            s->pending.pop_front();
            complete(s, r, BF_ERR_CANCELLED);
            continue;
        }
        const bf_fit_args &a = r->args;
        const size_t n = a.n, m = a.m, p = size_t(parameters(a.model));
        void *block = nullptr;
        cudaError_t e = inject ? cudaErrorMemoryAllocation : cudaMallocFromPoolAsync(&block, r->bytes, s->pool, s->copy);
        if (e == cudaErrorMemoryAllocation) {
            // The request fails alone: its bytes return to the budget and the
            // server goes on with the others.
            if (!inject)
                cudaGetLastError();
            s->pending.pop_front();
            complete(s, r, BF_ERR_CUDA);
            continue;
        }
        if (e != cudaSuccess) {
            report_cuda(e, "server allocation");
            return false;
        }
        r->block = static_cast<char *>(block);
        char *at = r->block;
        auto take = [&](size_t bytes) {
            char *here = at;
            at += align256(bytes);
            return here;
        };
        bf_fit_args d = a;
        d.memory = BF_MEMORY_DEVICE;
        d.x = reinterpret_cast<const float *>(take(m * 4));
        d.y = reinterpret_cast<const float *>(take(n * m * 4));
        d.p0 = a.p0 ? reinterpret_cast<const float *>(take(n * p * 4)) : nullptr;
        bf_fit_outputs o{};
        o.params = reinterpret_cast<float *>(take(n * p * 4));
        o.status = reinterpret_cast<int32_t *>(take(n * 4));
        o.iterations = reinterpret_cast<uint32_t *>(take(n * 4));
        o.chi2 = reinterpret_cast<float *>(take(n * 4));
        if (a.uncertainties) {
            o.covariance = reinterpret_cast<float *>(take(n * p * p * 4));
            o.standard_errors = reinterpret_cast<float *>(take(n * p * 4));
            o.uncertainty_status = reinterpret_cast<int32_t *>(take(n * 4));
        }
        r->guesses = reinterpret_cast<float *>(take(n * p * 4));
        r->counter = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long)));
        r->seg.args = d;
        r->seg.out = o;
        e = cudaMemcpyAsync(const_cast<float *>(d.x), a.x, m * 4, cudaMemcpyHostToDevice, s->copy);
        if (e == cudaSuccess && n)
            e = cudaMemcpyAsync(const_cast<float *>(d.y), a.y, n * m * 4, cudaMemcpyHostToDevice, s->copy);
        if (e == cudaSuccess && a.p0 && n)
            e = cudaMemcpyAsync(const_cast<float *>(d.p0), a.p0, n * p * 4, cudaMemcpyHostToDevice, s->copy);
        if (e != cudaSuccess) {
            report_cuda(e, "server copy-in");
            return false;
        }
        if (!mark) {
            mark = std::make_shared<CopyMark>();
            e = cudaEventCreateWithFlags(&mark->event, cudaEventDisableTiming);
            if (e != cudaSuccess) {
                report_cuda(e, "server copy-in event");
                return false;
            }
        }
        r->copied = mark;
        s->ready.push_back(r);
        s->pending.pop_front();
    }
    if (mark) {
        const cudaError_t e = cudaEventRecord(mark->event, s->copy);
        if (e != cudaSuccess) {
            report_cuda(e, "server copy-in event");
            return false;
        }
    }
    return true;
}

// Launch the ready requests (up to max_batch_fits) on a free slot.  Without
// allow_large, requests predicted to take longer than kBatchTargetMs stay queued:
// at most one slot runs a large request, so the other one is always free for
// short batches within a short batch's time.
bool launch(bf_server *s, Slot &slot, bool allow_large) {
    // Copies complete in admission order, so the requests whose inputs are on the
    // device are a prefix of the ready list: a batch never waits for other
    // requests' copies.
    //
    // Batches are kept short so that a small request never waits for a large one:
    // requests join in arrival order while the batch's predicted device time stays
    // within kBatchTargetMs; a request predicted to take longer runs alone (it starts
    // a batch, or waits for the next free slot), and later small requests may pass it.
    std::vector<std::shared_ptr<Request>> take;
    std::vector<bool> taken(s->ready.size(), false);
    uint64_t fits = 0;
    double predicted = 0.0;
    for (size_t i = 0; i < s->ready.size(); ++i) {
        const std::shared_ptr<Request> &r = s->ready[i];
        const uint64_t n = r->args.n;
        const double t = predicted_ms(r->args);
        const cudaError_t q = cudaEventQuery(r->copied->event);
        if (q == cudaErrorNotReady)
            break;
        if (q != cudaSuccess) {
            report_cuda(q, "server copy-in");
            return false;
        }
        if (!take.empty() && s->opt.max_batch_fits && fits + n > s->opt.max_batch_fits)
            break;
        if (!allow_large && t > kBatchTargetMs)
            continue; // waits for the other slot's large request to finish
        if (!take.empty() && predicted + t > kBatchTargetMs) {
            if (t > kBatchTargetMs)
                continue; // large: its own batch, later
            break;
        }
        take.push_back(r);
        taken[i] = true;
        fits += n;
        predicted += t;
        if (predicted > kBatchTargetMs)
            break; // a large request alone
    }
    if (take.empty())
        return true;
    size_t keep = 0;
    for (size_t i = 0; i < s->ready.size(); ++i)
        if (!taken[i])
            s->ready[keep++] = s->ready[i];
    s->ready.resize(keep);
    std::vector<bf_batch_segment> segs;
    segs.reserve(take.size());
    for (auto &r : take)
        segs.push_back(r->seg);
    cudaError_t e = cudaSuccess;
    bool launched = false;
    // A large batch's persistent kernels would hold every SM until its work drains,
    // and a short batch on the other slot could not start before.  With two slots a
    // large batch launches directly with grids for three quarters of the SMs' blocks,
    // which the hardware spreads over all SMs: every SM keeps room for the other
    // slot's blocks.
    const bool large = predicted > kBatchTargetMs;
    const bool shared = large && s->opt.max_in_flight != 1;
    const int sms = shared ? s->sms * 3 / 4 : s->sms;
    int rc = BF_OK;
    const bool direct = large && take.size() == 1 && bf::host::single_call_kernels_fit(take[0]->seg.args);
    if (direct) {
        // A large request alone runs the single-call kernels (rows staged in shared
        // memory, lanes per fit by (model, M)), as bf_cuda_fit would: faster per fit
        // than the batch kernels.
        const Request &r = *take[0];
        rc = bf::host::launch_single_call(r.seg.args, r.seg.out, r.guesses, r.counter, sms, slot.stream);
        slot.graph_used = false;
        launched = false; // no batch timing events
    } else {
        rc = bf::host::launch_planned(*slot.state, segs.data(), uint32_t(segs.size()),
                                      s->opt.batch_flags | (shared ? BF_BATCH_NO_GRAPH : 0u), sms, slot.stream,
                                      &launched, &slot.graph_used);
    }
    slot.launched = launched;
    if (rc != BF_OK) {
        // The batch could not be formed (a request failed validation on the device
        // path): complete its requests with the error, release their buffers.
        for (auto &r : take) {
            cudaFreeAsync(r->block, slot.stream);
            complete(s, r, rc);
        }
        return true;
    }
    if (e == cudaSuccess)
        e = cudaEventRecord(slot.done, slot.stream);
    if (e != cudaSuccess) {
        report_cuda(e, "server launch");
        return false;
    }
    slot.large = large;
    slot.requests = std::move(take);
    slot.busy = true;
    std::lock_guard<std::mutex> lock(s->mutex);
    s->stats.batches += launched || direct ? 1 : 0;
    s->stats.max_batch_requests = std::max<uint64_t>(s->stats.max_batch_requests, slot.requests.size());
    return true;
}

// Retire a slot whose batch finished: outputs back to the callers' host buffers
// (issued only now, because a copy into pageable memory would block the scheduler
// until the batch ends), device memory back to the pool.  False on a CUDA failure.
bool retire(bf_server *s, Slot &slot) {
    const cudaError_t q = cudaEventQuery(slot.done);
    if (q == cudaErrorNotReady)
        return true;
    if (q != cudaSuccess) {
        report_cuda(q, "server batch");
        return false;
    }
    bf_cuda_timing t{};
    if (slot.launched && bf::host::finish_planned(*slot.state, slot.graph_used, &t) == BF_OK) {
        std::lock_guard<std::mutex> lock(s->mutex);
        s->stats.gpu_ms += t.kernel_ms;
    }
    cudaError_t e = cudaSuccess;
    for (auto &r : slot.requests) {
        const bf_fit_args &a = r->args;
        const size_t n = a.n, p = size_t(parameters(a.model));
        const bf_fit_outputs &d = r->seg.out, &h = r->host_out;
        auto back = [&](void *dst, const void *src, size_t bytes) {
            if (e == cudaSuccess && bytes)
                e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, slot.stream);
        };
        back(h.params, d.params, n * p * 4);
        back(h.status, d.status, n * 4);
        back(h.iterations, d.iterations, n * 4);
        back(h.chi2, d.chi2, n * 4);
        if (a.uncertainties) {
            back(h.covariance, d.covariance, n * p * p * 4);
            back(h.standard_errors, d.standard_errors, n * p * 4);
            back(h.uncertainty_status, d.uncertainty_status, n * 4);
        }
        if (e == cudaSuccess)
            e = cudaFreeAsync(r->block, slot.stream);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(slot.stream);
    if (e != cudaSuccess) {
        report_cuda(e, "server copy-out");
        return false;
    }
    for (auto &r : slot.requests)
        complete(s, r, BF_OK);
    slot.requests.clear();
    slot.busy = false;
    return true;
}

void fail_everything(bf_server *s, const std::string &why) {
    std::vector<std::shared_ptr<Request>> all;
    for (auto &slot : s->slot) {
        for (auto &r : slot.requests)
            all.push_back(r);
        slot.requests.clear();
        slot.busy = false;
    }
    for (auto &r : s->ready)
        all.push_back(r);
    s->ready.clear();
    for (auto &r : s->pending)
        all.push_back(r);
    s->pending.clear();
    {
        std::lock_guard<std::mutex> lock(s->mutex);
        s->fatal = why;
        for (auto &r : s->incoming)
            all.push_back(r);
        s->incoming.clear();
    }
    for (auto &r : all)
        complete(s, r, BF_ERR_CUDA);
}

void scheduler(bf_server *s) {
    cudaSetDevice(s->device);
    const int slots = s->opt.max_in_flight == 1 ? 1 : 2;
    while (true) {
        bool stop = false;
        {
            std::unique_lock<std::mutex> lock(s->mutex);
            const bool running = s->slot[0].busy || s->slot[1].busy;
            const bool work = !s->ready.empty() || !s->pending.empty();
            if (!running && !work && s->incoming.empty() && !s->stopping)
                s->wake.wait(lock, [&] { return !s->incoming.empty() || s->stopping; });
            else if (s->incoming.empty())
                s->wake.wait_for(lock, std::chrono::microseconds(50)); // poll copies and batches
            while (!s->incoming.empty()) {
                s->pending.push_back(std::move(s->incoming.front()));
                s->incoming.pop_front();
            }
            stop = s->stopping && s->pending.empty() && s->ready.empty() && !s->slot[0].busy && !s->slot[1].busy;
        }
        if (stop)
            return;
        bool ok = true;
        for (int i = 0; i < slots && ok; ++i)
            if (s->slot[i].busy)
                ok = retire(s, s->slot[i]);
        if (ok)
            ok = admit(s);
        for (int i = 0; i < slots && ok && !s->ready.empty(); ++i)
            if (!s->slot[i].busy) {
                // With two slots, a large request may take a slot only while the
                // other one is not running one.
                const bool other_large = slots == 2 && s->slot[1 - i].busy && s->slot[1 - i].large;
                ok = launch(s, s->slot[i], !other_large);
            }
        if (!ok) {
            fail_everything(s, bf_cuda_last_error());
            return;
        }
    }
}

void destroy(bf_server *s) {
    for (auto &slot : s->slot) {
        if (slot.stream)
            cudaStreamSynchronize(slot.stream);
        bf::host::release_batch_state(slot.state);
        if (slot.done)
            cudaEventDestroy(slot.done);
        if (slot.stream)
            cudaStreamDestroy(slot.stream);
    }
    if (s->copy) {
        cudaStreamSynchronize(s->copy);
        cudaStreamDestroy(s->copy);
    }
    if (s->pool)
        cudaMemPoolDestroy(s->pool);
    delete s;
}

} // namespace

extern "C" {

int bf_server_create(int device, const bf_server_options *options, bf_server **out) {
    if (!out)
        return report(BF_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (options && options->max_in_flight > 2)
        return report(BF_ERR_INVALID_ARGUMENT, "max_in_flight must be 0, 1 or 2");
    if (options && (options->batch_flags & ~(BF_BATCH_FIXED_MAPPING | BF_BATCH_NO_GRAPH)))
        return report(BF_ERR_INVALID_ARGUMENT, "unknown batch flags");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return report(BF_ERR_UNAVAILABLE, "CUDA fitting is unavailable: no CUDA device");
    if (device < 0 || device >= count)
        return report(BF_ERR_INVALID_ARGUMENT, "device index out of range");
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess)
        return report_cuda(e, "cudaGetDeviceProperties");
    if (prop.major != 10)
        return report(BF_ERR_UNAVAILABLE, "CUDA fitting is unavailable: the device is not sm_100");
    auto *s = new bf_server();
    s->device = device;
    s->sms = prop.multiProcessorCount;
    if (options)
        s->opt = *options;
    e = cudaSetDevice(device);
    size_t free_bytes = 0, total_bytes = 0;
    if (e == cudaSuccess)
        e = cudaMemGetInfo(&free_bytes, &total_bytes);
    const uint64_t cap = 150ull << 30;
    uint64_t budget = s->opt.memory_budget ? s->opt.memory_budget : cap;
    const uint64_t reserve = 2ull << 30; // batch arenas, graphs and the CUDA runtime
    budget = std::min<uint64_t>(budget, free_bytes > reserve ? free_bytes - reserve : free_bytes / 2);
    s->stats.memory_budget = budget;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (e == cudaSuccess)
        e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        uint64_t keep = budget; // freed blocks stay in the pool for the next requests
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
    // Map pool memory now (up to 8 GB of the budget): growing the pool while requests
    // arrive would stall admission for milliseconds per growth.
    if (e == cudaSuccess) {
        void *warm = nullptr;
        const size_t bytes = size_t(std::min<uint64_t>(budget, 8ull << 30));
        e = cudaMallocFromPoolAsync(&warm, bytes, s->pool, s->copy);
        if (e == cudaSuccess)
            e = cudaFreeAsync(warm, s->copy);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s->copy);
    }
    for (auto &slot : s->slot) {
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
        if (e == cudaSuccess && bf::host::create_batch_state(&slot.state) != BF_OK)
            e = cudaErrorMemoryAllocation;
        // Arena and graph sized up front: a batch within these sizes allocates
        // nothing and never synchronises the device.
        const uint64_t fits = s->opt.max_batch_fits ? s->opt.max_batch_fits : (4ull << 20);
        if (e == cudaSuccess &&
            bf::host::prepare_planned(*slot.state, 16384, size_t(fits), s->sms, slot.stream) != BF_OK)
            e = cudaErrorMemoryAllocation;
    }
    if (e != cudaSuccess) {
        destroy(s);
        return report_cuda(e, "server setup");
    }
    s->worker = std::thread(scheduler, s);
    *out = s;
    return BF_OK;
}

void bf_server_destroy(bf_server *s) {
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> lock(s->mutex);
        s->stopping = true;
    }
    s->wake.notify_all();
    if (s->worker.joinable())
        s->worker.join();
    destroy(s);
}

int bf_server_submit(bf_server *s, const bf_fit_args *args, const bf_fit_outputs *out, uint64_t *ticket) {
    if (!s || !args || !out || !ticket)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    if (args->memory != BF_MEMORY_HOST)
        return report(BF_ERR_INVALID_ARGUMENT, "server requests take host memory");
    bf::FitArgs base{};
    int rc = bf::host::prepare_segment(args, out, uint32_t(bf::kBatchMaxPoints), &base);
    if (rc != BF_OK)
        return rc;
    if (args->n > uint64_t(0x7fffffff))
        return report(BF_ERR_INVALID_ARGUMENT, "more than 2^31-1 fits in one request");
    auto r = std::make_shared<Request>();
    r->args = *args;
    r->host_out = *out;
    r->bytes = request_bytes(*args);
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mutex);
        if (!s->fatal.empty())
            return report(BF_ERR_CUDA, "server stopped after a CUDA failure: " + s->fatal);
        if (s->stopping)
            return report(BF_ERR_INVALID_ARGUMENT, "server is shutting down");
        if (r->bytes > s->stats.memory_budget)
            return report(BF_ERR_INVALID_ARGUMENT, "request needs " + std::to_string(r->bytes) +
                                                       " device bytes, more than the server's budget of " +
                                                       std::to_string(s->stats.memory_budget));
        r->ticket = s->next_ticket++;
        s->tickets[r->ticket] = r;
        s->stats.submitted += 1;
        s->incoming.push_back(r);
        *ticket = r->ticket;
    }
    s->wake.notify_one();
    return BF_OK;
}

int bf_server_poll(bf_server *s, uint64_t ticket) {
    if (!s)
        return -BF_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mutex);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return -BF_ERR_INVALID_ARGUMENT;
    return it->second->finished ? 1 : 0;
}

int bf_server_wait(bf_server *s, uint64_t ticket, double *latency_ms) {
    if (!s)
        return report(BF_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lock(s->mutex);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return report(BF_ERR_INVALID_ARGUMENT, "unknown ticket");
    std::shared_ptr<Request> r = it->second;
    s->finished.wait(lock, [&] { return r->finished; });
    s->tickets.erase(ticket);
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->done - r->submitted).count();
    if (r->result != BF_OK)
        return report(r->result, s->fatal.empty() ? "request failed" : "request failed: " + s->fatal);
    return BF_OK;
}

int bf_server_cancel(bf_server *s, uint64_t ticket) {
    if (!s)
        return -BF_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mutex);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return -BF_ERR_INVALID_ARGUMENT;
    Request &r = *it->second;
    if (r.finished || r.charged || r.cancelled)
        return r.cancelled ? 1 : 0;
    r.cancelled = true; // the scheduler completes it before admission
    s->wake.notify_one();
    return 1;
}

int bf_server_fail_allocations(bf_server *s, uint32_t count) {
    if (!s)
        return report(BF_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lock(s->mutex);
    s->fail_allocations = count;
    return BF_OK;
}

int bf_server_get_stats(bf_server *s, bf_server_stats *out) {
    if (!s || !out)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mutex);
    *out = s->stats;
    return BF_OK;
}

} // extern "C"
