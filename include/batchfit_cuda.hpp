// batchfit_cuda.hpp -- header-only C++ API of the batchfit B200 backend, over the
// C ABI in batchfit_cuda.h.
//
// It mirrors the reference's batch API (include/batchfit/metal/batch.hpp:160-310)
// so that a C++ caller moves from the Metal device to CUDA by swapping names:
//
//   reference (batchfit::)                      here (batchfit::cuda::)
//   metal::Context::make_batch<Model>(n, m, u)  Context::make_batch<Model>(n, m, u)
//   metal::SharedBatch  x() y() initial()       SharedBatch  x() y() initial()
//     fits() points() capacity() resize_fits()    (same; y is fit-major, y[i*M+m])
//   fit_batch<Model>(batch, Device::Metal,      fit_batch<Model>(batch, options,
//                    options, variant)                           variant)
//   submit_batch<Model>(batch, options, v)      submit_batch<Model>(batch, options, v)
//   metal::PendingBatch{ready(), get()}         PendingBatch{ready(), get()}
//   metal::Result (spans, timings)              Result (spans, timings)
//   cpu::SolverOptions<float, P>                SolverOptions<P>
//   models::Gaussian / Lorentzian /             Gaussian / Lorentzian /
//     PseudoVoigt / TwoLorentzian                 PseudoVoigt / TwoLorentzian (tags)
//   metal::KernelVariant                        KernelVariant (lanes per fit)
//   FitStatus, UncertaintyStatus                FitStatus, UncertaintyStatus (same codes)
//
// Errors follow the reference: bad arguments throw std::invalid_argument, CUDA and
// device failures std::runtime_error, touching a batch while it is in flight
// std::logic_error.  Per-fit failures are statuses, never exceptions.
//
// Link with batchfit_b200/libbatchfit_cuda.so.
#pragma once

#include "batchfit_cuda.h"

#include <array>
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <mutex>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace batchfit {
namespace cuda {

// Status codes equal the reference's (solver.hpp:16-23, uncertainty_types.hpp:3-10).
enum class FitStatus : int32_t {
    converged,
    max_iterations,
    singular_matrix,
    invalid_input,
    degenerate_data,
    unresolved_peak
};
enum class UncertaintyStatus : int32_t {
    available,
    not_converged,
    insufficient_dof,
    singular_matrix,
    active_bound,
    invalid_input
};

// Model tags: parameter order as the reference's models (models.hpp:78-185).
struct Gaussian {
    static constexpr int32_t id = BF_MODEL_GAUSSIAN;
    static constexpr std::size_t parameter_count = 3;
};
struct Lorentzian {
    static constexpr int32_t id = BF_MODEL_LORENTZIAN;
    static constexpr std::size_t parameter_count = 3;
};
struct PseudoVoigt {
    static constexpr int32_t id = BF_MODEL_PSEUDO_VOIGT;
    static constexpr std::size_t parameter_count = 4;
};
struct TwoLorentzian {
    static constexpr int32_t id = BF_MODEL_TWO_LORENTZIAN;
    static constexpr std::size_t parameter_count = 8;
};

// The mapping of fits to the GPU (the reference's KernelVariant chooses thread,
// SIMD-group or threadgroup per fit): Automatic picks by model and M.
enum class KernelVariant { Automatic, GroupOf8, GroupOf16, GroupOf32, CtaPerFit };
enum class Policy : uint32_t { Reference = BF_POLICY_REFERENCE, Parity = BF_POLICY_PARITY };

// cpu::SolverOptions<float, P> (solver.hpp:26-41) plus the stopping policy.  The
// tolerances default to the policy's (bf_cuda_default_options).
template <std::size_t P> struct SolverOptions {
    Policy policy = Policy::Parity;
    unsigned max_iterations = 100;
    double initial_lambda = 1e-3;
    double gradient_tolerance = -1, step_tolerance = -1, cost_tolerance = -1; // < 0: the policy's default
    bool compensated_sum = false;
    bool scaled_cholesky = false;
    std::array<float, P> lower;
    std::array<float, P> upper;
    SolverOptions() {
        lower.fill(-std::numeric_limits<float>::infinity());
        upper.fill(std::numeric_limits<float>::infinity());
    }
};

struct Timings {
    double gpu_seconds = 0, wall_seconds = 0;
    double guess_seconds = 0, lm_seconds = 0, covariance_seconds = 0;
    int lanes_per_fit = 0, grid = 0, blocks_per_sm = 0;
    KernelVariant variant = KernelVariant::Automatic;
};

namespace detail {

[[noreturn]] inline void raise(int rc, const char *what) {
    const std::string message = std::string(what) + ": " + bf_cuda_last_error();
    if (rc == BF_ERR_INVALID_ARGUMENT)
        throw std::invalid_argument(message);
    if (rc == BF_ERR_BUSY)
        throw std::logic_error(message);
    throw std::runtime_error(message);
}

inline void check(int rc, const char *what) {
    if (rc != BF_OK)
        raise(rc, what);
}

inline int32_t lanes_of(KernelVariant v) {
    switch (v) {
    case KernelVariant::GroupOf8: return 8;
    case KernelVariant::GroupOf16: return 16;
    case KernelVariant::GroupOf32: return 32;
    case KernelVariant::CtaPerFit: return 128;
    default: return 0;
    }
}

inline KernelVariant variant_of(int32_t lanes) {
    switch (lanes) {
    case 8: return KernelVariant::GroupOf8;
    case 16: return KernelVariant::GroupOf16;
    case 32: return KernelVariant::GroupOf32;
    case 128: return KernelVariant::CtaPerFit;
    default: return KernelVariant::Automatic;
    }
}

// Host buffer in pinned memory when the library can provide it (copies then
// overlap the kernels), in pageable memory otherwise.
template <class T> class HostArray {
  public:
    HostArray() = default;
    explicit HostArray(std::size_t n) : size_(n) {
        if (n == 0)
            return;
        void *p = nullptr;
        if (bf_cuda_host_alloc(n * sizeof(T), &p) == BF_OK && p) {
            data_ = static_cast<T *>(p);
            pinned_ = true;
        } else {
            data_ = new T[n]();
        }
    }
    HostArray(const HostArray &) = delete;
    HostArray &operator=(const HostArray &) = delete;
    HostArray(HostArray &&other) noexcept { *this = std::move(other); }
    HostArray &operator=(HostArray &&other) noexcept {
        if (this != &other) {
            free();
            data_ = std::exchange(other.data_, nullptr);
            size_ = std::exchange(other.size_, 0);
            pinned_ = std::exchange(other.pinned_, false);
        }
        return *this;
    }
    ~HostArray() { free(); }
    T *data() const { return data_; }
    std::size_t size() const { return size_; }

  private:
    void free() {
        if (pinned_)
            bf_cuda_host_free(data_);
        else
            delete[] data_;
        data_ = nullptr;
    }
    T *data_ = nullptr;
    std::size_t size_ = 0;
    bool pinned_ = false;
};

// The C ABI contexts of one Context: each serialises its calls and holds one
// submission at a time, so concurrent submissions take one each.
class ContextPool {
  public:
    explicit ContextPool(int device) : device_(device) { release(acquire()); }
    ~ContextPool() {
        for (bf_cuda_context *c : free_)
            bf_cuda_context_destroy(c);
    }
    bf_cuda_context *acquire() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            if (!free_.empty()) {
                bf_cuda_context *c = free_.back();
                free_.pop_back();
                return c;
            }
        }
        bf_cuda_context *c = nullptr;
        check(bf_cuda_context_create(device_, &c), "bf_cuda_context_create");
        return c;
    }
    void release(bf_cuda_context *c) {
        std::lock_guard<std::mutex> lock(mutex_);
        free_.push_back(c);
    }

  private:
    int device_;
    std::mutex mutex_;
    std::vector<bf_cuda_context *> free_;
};

struct Storage {
    std::size_t fits = 0, capacity = 0, points = 0, p = 0;
    int32_t model = 0;
    bool uncertainties = false;
    HostArray<float> x, y, initial, parameters, chi_squared, covariance, standard_errors;
    HostArray<int32_t> status, uncertainty_status;
    HostArray<uint32_t> iterations;
    std::shared_ptr<ContextPool> pool;
    std::atomic<bool> busy{false};
    bool has_initial = true; // false: data-only guesses (initial values are ignored)
};

struct BusyLease {
    explicit BusyLease(Storage &value) : storage(value) {
        if (storage.busy.exchange(true))
            throw std::logic_error("CUDA batch is already in flight");
    }
    ~BusyLease() {
        if (active)
            storage.busy.store(false);
    }
    BusyLease(const BusyLease &) = delete;
    BusyLease &operator=(const BusyLease &) = delete;
    Storage &storage;
    bool active = true;
};

template <class Model>
inline bf_fit_args make_args(const Storage &s, const SolverOptions<Model::parameter_count> &o, KernelVariant v) {
    bf_fit_args a{};
    a.model = Model::id;
    a.n = s.fits;
    a.m = uint32_t(s.points);
    a.x = s.x.data();
    a.y = s.y.data();
    a.p0 = s.has_initial ? s.initial.data() : nullptr;
    a.memory = BF_MEMORY_HOST;
    a.uncertainties = s.uncertainties ? 1 : 0;
    a.group_lanes = lanes_of(v);
    check(bf_cuda_default_options(Model::id, uint32_t(o.policy), &a.options), "bf_cuda_default_options");
    a.options.max_iterations = o.max_iterations;
    a.options.initial_lambda = o.initial_lambda;
    if (o.gradient_tolerance >= 0)
        a.options.gradient_tolerance = o.gradient_tolerance;
    if (o.step_tolerance >= 0)
        a.options.step_tolerance = o.step_tolerance;
    if (o.cost_tolerance >= 0)
        a.options.cost_tolerance = o.cost_tolerance;
    a.options.compensated_sum = o.compensated_sum ? 1u : 0u;
    a.options.scaled_cholesky = o.scaled_cholesky ? 1u : 0u;
    for (std::size_t k = 0; k < Model::parameter_count; ++k) {
        a.options.lower[k] = o.lower[k];
        a.options.upper[k] = o.upper[k];
    }
    a.y_format = BF_Y_FLOAT32;
    return a;
}

inline bf_fit_outputs make_outputs(Storage &s) {
    bf_fit_outputs out{};
    out.params = s.parameters.data();
    out.status = s.status.data();
    out.iterations = s.iterations.data();
    out.chi2 = s.chi_squared.data();
    if (s.uncertainties) {
        out.covariance = s.covariance.data();
        out.standard_errors = s.standard_errors.data();
        out.uncertainty_status = s.uncertainty_status.data();
    }
    return out;
}

inline Timings timings_of(bf_cuda_context *c, double wall_seconds) {
    bf_cuda_timing t{};
    check(bf_cuda_last_timing(c, &t), "bf_cuda_last_timing");
    Timings r;
    r.gpu_seconds = t.kernel_ms * 1e-3;
    r.wall_seconds = wall_seconds;
    r.guess_seconds = t.guess_ms * 1e-3;
    r.lm_seconds = t.lm_ms * 1e-3;
    r.covariance_seconds = t.covariance_ms * 1e-3;
    r.lanes_per_fit = t.group_lanes;
    r.grid = t.grid;
    r.blocks_per_sm = t.blocks_per_sm;
    r.variant = variant_of(t.group_lanes);
    return r;
}

struct Access;
struct PendingAccess;
} // namespace detail

inline bool available() { return bf_cuda_available() != 0; }

class SharedBatch {
  public:
    std::size_t fits() const { return storage_->fits; }
    std::size_t points() const { return storage_->points; }
    std::size_t capacity() const { return storage_->capacity; }
    std::span<float> x() {
        ensure_idle();
        return {storage_->x.data(), storage_->points};
    }
    // Fit-major: y[i*M+m] (the Metal batch is point-major; no transpose is needed here).
    std::span<float> y() {
        ensure_idle();
        return {storage_->y.data(), storage_->fits * storage_->points};
    }
    // Fit-major: initial[i*P+k].
    std::span<float> initial() {
        ensure_idle();
        return {storage_->initial.data(), storage_->fits * storage_->p};
    }
    // With false, the fit starts from data-only guesses on the GPU (the reference's
    // Python binding runs cpu::initial_guess per row first) and initial() is ignored.
    void use_initial(bool given) {
        detail::BusyLease lease(*storage_);
        storage_->has_initial = given;
    }
    void resize_fits(std::size_t fits) {
        detail::BusyLease lease(*storage_);
        if (fits > storage_->capacity)
            throw std::out_of_range("CUDA active fits exceed buffer capacity");
        storage_->fits = fits;
    }

  private:
    void ensure_idle() const {
        if (storage_->busy.load())
            throw std::logic_error("CUDA input access while batch is in flight");
    }
    explicit SharedBatch(std::shared_ptr<detail::Storage> storage) : storage_(std::move(storage)) {}
    std::shared_ptr<detail::Storage> storage_;
    friend class Context;
    friend struct detail::Access;
};

struct detail::Access {
    static std::shared_ptr<Storage> owner(SharedBatch &batch) { return batch.storage_; }
};

struct Result {
    std::span<const float> parameters;
    std::span<const FitStatus> status;
    std::span<const unsigned> iterations;
    std::span<const float> chi_squared;
    Timings timings;
    std::span<const float> covariance, standard_errors;
    std::span<const UncertaintyStatus> uncertainty_status;
    bool has_uncertainties = false;

    Result(std::shared_ptr<detail::Storage> storage, Timings times)
        : parameters(storage->parameters.data(), storage->fits * storage->p),
          status(reinterpret_cast<const FitStatus *>(storage->status.data()), storage->fits),
          iterations(storage->iterations.data(), storage->fits),
          chi_squared(storage->chi_squared.data(), storage->fits), timings(times),
          has_uncertainties(storage->uncertainties), owner_(std::move(storage)) {
        if (has_uncertainties) {
            const auto &s = *owner_;
            covariance = {s.covariance.data(), s.fits * s.p * s.p};
            standard_errors = {s.standard_errors.data(), s.fits * s.p};
            uncertainty_status = {reinterpret_cast<const UncertaintyStatus *>(s.uncertainty_status.data()), s.fits};
        }
    }

  private:
    std::shared_ptr<detail::Storage> owner_;
};

class Context {
  public:
    // The first sm_100 device unless another is named; std::runtime_error when
    // CUDA fitting is unavailable.
    explicit Context(int device = 0) : pool_(std::make_shared<detail::ContextPool>(device)) {}

    template <class Model> SharedBatch make_batch(std::size_t n, std::size_t m, bool uncertainties = false) const {
        constexpr std::size_t p = Model::parameter_count;
        if (m == 0)
            throw std::invalid_argument("CUDA batch requires nonempty x[M] (M > 0)");
        if (m > bf_cuda_max_points(Model::id))
            throw std::invalid_argument("CUDA batch M exceeds the backend's limit");
        if (n > (SIZE_MAX / sizeof(float)) / (m + p * p))
            throw std::invalid_argument("CUDA batch size overflows");
        auto s = std::make_shared<detail::Storage>();
        s->fits = s->capacity = n;
        s->points = m;
        s->p = p;
        s->model = Model::id;
        s->uncertainties = uncertainties;
        s->x = detail::HostArray<float>(m);
        s->y = detail::HostArray<float>(n * m);
        s->initial = detail::HostArray<float>(n * p);
        s->parameters = detail::HostArray<float>(n * p);
        s->status = detail::HostArray<int32_t>(n);
        s->iterations = detail::HostArray<uint32_t>(n);
        s->chi_squared = detail::HostArray<float>(n);
        if (uncertainties) {
            s->covariance = detail::HostArray<float>(n * p * p);
            s->standard_errors = detail::HostArray<float>(n * p);
            s->uncertainty_status = detail::HostArray<int32_t>(n);
        }
        s->pool = pool_;
        return SharedBatch(std::move(s));
    }

  private:
    std::shared_ptr<detail::ContextPool> pool_;
};

class PendingBatch {
  public:
    PendingBatch(PendingBatch &&other) noexcept { *this = std::move(other); }
    PendingBatch &operator=(PendingBatch &&other) noexcept {
        if (this != &other) {
            drain();
            owner_ = std::move(other.owner_);
            context_ = std::exchange(other.context_, nullptr);
            pending_ = std::exchange(other.pending_, nullptr);
            start_ = other.start_;
        }
        return *this;
    }
    PendingBatch(const PendingBatch &) = delete;
    PendingBatch &operator=(const PendingBatch &) = delete;
    // An uncollected submission is waited for (its outputs still land in the batch).
    ~PendingBatch() { drain(); }

    bool ready() const {
        if (!pending_)
            throw std::logic_error("CUDA pending batch was already collected");
        const int r = bf_cuda_ready(pending_);
        if (r < 0)
            detail::raise(-r, "bf_cuda_ready");
        return r == 1;
    }
    // Waits, then returns the results or rethrows the submission's error.
    Result get() {
        if (!pending_)
            throw std::logic_error("CUDA pending batch was already collected");
        const int rc = bf_cuda_wait(std::exchange(pending_, nullptr));
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count();
        auto owner = std::move(owner_);
        bf_cuda_context *context = std::exchange(context_, nullptr);
        owner->busy.store(false);
        if (rc != BF_OK) {
            owner->pool->release(context);
            detail::raise(rc, "bf_cuda_submit");
        }
        Timings t;
        try {
            t = detail::timings_of(context, wall);
        } catch (...) {
            owner->pool->release(context);
            throw;
        }
        owner->pool->release(context);
        return Result(std::move(owner), t);
    }

  private:
    PendingBatch(std::shared_ptr<detail::Storage> owner, bf_cuda_context *context, bf_cuda_pending *pending,
                 std::chrono::steady_clock::time_point start)
        : owner_(std::move(owner)), context_(context), pending_(pending), start_(start) {}
    void drain() noexcept {
        if (pending_) {
            bf_cuda_wait(std::exchange(pending_, nullptr));
            owner_->busy.store(false);
            owner_->pool->release(std::exchange(context_, nullptr));
        }
    }
    std::shared_ptr<detail::Storage> owner_;
    bf_cuda_context *context_ = nullptr;
    bf_cuda_pending *pending_ = nullptr;
    std::chrono::steady_clock::time_point start_{};
    friend struct detail::PendingAccess;
};

struct detail::PendingAccess {
    static PendingBatch make(std::shared_ptr<Storage> owner, bf_cuda_context *context, bf_cuda_pending *pending,
                             std::chrono::steady_clock::time_point start) {
        return PendingBatch(std::move(owner), context, pending, start);
    }
};

// submit_batch<Model> (include/batchfit/metal/batch.hpp:253-264): queues the fit
// and returns at once; the batch stays in flight (its spans refuse access) until
// get() or the PendingBatch's destruction.
template <class Model>
PendingBatch submit_batch(SharedBatch &batch, const SolverOptions<Model::parameter_count> &options = {},
                          KernelVariant variant = KernelVariant::Automatic) {
    auto owner = detail::Access::owner(batch);
    if (owner->model != Model::id)
        throw std::invalid_argument("CUDA batch/model parameter count mismatch");
    detail::BusyLease lease(*owner);
    const bf_fit_args args = detail::make_args<Model>(*owner, options, variant);
    const bf_fit_outputs out = detail::make_outputs(*owner);
    const auto start = std::chrono::steady_clock::now();
    bf_cuda_context *context = owner->pool->acquire();
    bf_cuda_pending *pending = nullptr;
    const int rc = bf_cuda_submit(context, &args, &out, &pending);
    if (rc != BF_OK) {
        owner->pool->release(context);
        detail::raise(rc, "bf_cuda_submit");
    }
    lease.active = false;
    return detail::PendingAccess::make(std::move(owner), context, pending, start);
}

// fit_batch<Model> (include/batchfit/metal/batch.hpp:268-310) with the CUDA device:
// fits every row of the batch and returns spans over its outputs.
template <class Model>
Result fit_batch(SharedBatch &batch, const SolverOptions<Model::parameter_count> &options = {},
                 KernelVariant variant = KernelVariant::Automatic) {
    return submit_batch<Model>(batch, options, variant).get();
}

} // namespace cuda
} // namespace batchfit
