// Checks of the header-only C++ API (include/batchfit_cuda.hpp), run by
// tests/test_cpp_api.py:
//   twin_check cpu  -- on a machine without an sm_100 GPU: the API reports the
//                      device unavailable with std::runtime_error
//   twin_check gpu  -- fit_batch / submit_batch on a pseudo-Voigt batch: results
//                      equal the C ABI's bit for bit, in-flight access throws
//                      std::logic_error, bad arguments std::invalid_argument, and
//                      two batches can be in flight on one Context.
// Prints OK on success; any failure prints FAIL and exits 1.
#include "batchfit_cuda.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace bc = batchfit::cuda;

static int failures = 0;
#define CHECK(cond)                                                                                    \
    do {                                                                                               \
        if (!(cond)) {                                                                                 \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #cond);                                 \
            ++failures;                                                                                \
        }                                                                                              \
    } while (0)

template <class E, class F> static bool throws(F &&f) {
    try {
        f();
    } catch (const E &) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

// Seeded pseudo-Voigt spectra on x = linspace(-10, 10, m).
static void fill(bc::SharedBatch &b, unsigned seed) {
    auto x = b.x();
    const std::size_t m = x.size();
    for (std::size_t j = 0; j < m; ++j)
        x[j] = float(-10.0 + 20.0 * double(j) / double(m - 1));
    auto y = b.y();
    unsigned long long s = 0x9e3779b97f4a7c15ull ^ seed;
    auto uniform = [&s] {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return double(s >> 11) * 0x1.0p-53;
    };
    for (std::size_t i = 0; i < b.fits(); ++i) {
        const double a = 0.5 + 4.5 * uniform(), c = -6 + 12 * uniform(), w = 0.3 + 2 * uniform(), eta = uniform();
        for (std::size_t j = 0; j < m; ++j) {
            const double z = (x[j] - c) / w;
            const double clean = a * ((1 - eta) * std::exp(-4 * std::log(2.0) * z * z) + eta / (1 + 4 * z * z));
            const double noise = 0.01 * a * (uniform() + uniform() + uniform() - 1.5) * 2.0;
            y[i * m + j] = float(clean + noise);
        }
    }
}

static int cpu_mode() {
    CHECK(!bc::available());
    CHECK(throws<std::runtime_error>([] { bc::Context ctx; }));
    return 0;
}

static int gpu_mode() {
    CHECK(bc::available());
    bc::Context ctx;
    const std::size_t n = 3000, m = 512;
    auto batch = ctx.make_batch<bc::PseudoVoigt>(n, m, true);
    fill(batch, 1);
    batch.use_initial(false);
    bc::SolverOptions<4> opts;
    opts.lower = {0.0f, -10.0f, 1e-3f, 0.0f};
    opts.upper = {INFINITY, 10.0f, 10.0f, 1.0f};
    bc::Result r = bc::fit_batch<bc::PseudoVoigt>(batch, opts);
    CHECK(r.parameters.size() == n * 4 && r.status.size() == n && r.has_uncertainties);
    std::size_t converged = 0;
    for (auto st : r.status)
        converged += st == bc::FitStatus::converged;
    CHECK(converged >= n * 95 / 100);
    CHECK(r.timings.gpu_seconds > 0 && r.timings.wall_seconds > 0);

    // The same fit through the C ABI: equal bit for bit.
    bf_cuda_context *c = nullptr;
    CHECK(bf_cuda_context_create(0, &c) == BF_OK);
    bf_fit_args a{};
    a.model = BF_MODEL_PSEUDO_VOIGT;
    a.n = n;
    a.m = m;
    a.x = batch.x().data();
    a.y = batch.y().data();
    a.p0 = nullptr;
    a.memory = BF_MEMORY_HOST;
    a.uncertainties = 1;
    CHECK(bf_cuda_default_options(BF_MODEL_PSEUDO_VOIGT, BF_POLICY_PARITY, &a.options) == BF_OK);
    for (int k = 0; k < 4; ++k) {
        a.options.lower[k] = opts.lower[k];
        a.options.upper[k] = opts.upper[k];
    }
    std::vector<float> params(n * 4), chi2(n), cov(n * 16), se(n * 4);
    std::vector<int32_t> status(n), ustatus(n);
    std::vector<uint32_t> iters(n);
    bf_fit_outputs o{params.data(), status.data(), iters.data(), chi2.data(), cov.data(), se.data(), ustatus.data()};
    CHECK(bf_cuda_fit(c, &a, &o) == BF_OK);
    bf_cuda_context_destroy(c);
    CHECK(std::memcmp(params.data(), r.parameters.data(), n * 4 * sizeof(float)) == 0);
    CHECK(std::memcmp(chi2.data(), r.chi_squared.data(), n * sizeof(float)) == 0);
    CHECK(std::memcmp(status.data(), r.status.data(), n * sizeof(int32_t)) == 0);
    CHECK(std::memcmp(cov.data(), r.covariance.data(), n * 16 * sizeof(float)) == 0);

    // Asynchronous: the batch refuses access while in flight; two batches in flight.
    auto second = ctx.make_batch<bc::PseudoVoigt>(n, m, false);
    fill(second, 2);
    second.use_initial(false);
    bc::PendingBatch p1 = bc::submit_batch<bc::PseudoVoigt>(batch, opts);
    bc::PendingBatch p2 = bc::submit_batch<bc::PseudoVoigt>(second, opts);
    CHECK(throws<std::logic_error>([&] { batch.y(); }));
    CHECK(throws<std::logic_error>([&] { bc::submit_batch<bc::PseudoVoigt>(batch, opts); }));
    bc::Result r1 = p1.get();
    bc::Result r2 = p2.get();
    CHECK(std::memcmp(params.data(), r1.parameters.data(), n * 4 * sizeof(float)) == 0);
    CHECK(r2.status.size() == n && !r2.has_uncertainties);
    CHECK(throws<std::logic_error>([&] { p1.get(); }));
    {
        bc::PendingBatch dropped = bc::submit_batch<bc::PseudoVoigt>(second, opts);
    } // drained by its destructor
    CHECK(!throws<std::logic_error>([&] { second.y(); }));

    // Bad arguments.
    CHECK(throws<std::invalid_argument>([&] { ctx.make_batch<bc::Gaussian>(4, 0); }));
    CHECK(throws<std::invalid_argument>([&] { bc::fit_batch<bc::Gaussian>(batch); }));
    // Per-fit failures are statuses: invalid bounds give invalid_input, no exception.
    bc::SolverOptions<4> bad = opts;
    bad.lower[0] = 2.0f;
    bad.upper[0] = 1.0f;
    bc::Result rb = bc::fit_batch<bc::PseudoVoigt>(batch, bad);
    CHECK(rb.status[0] == bc::FitStatus::invalid_input);
    // The CTA-per-fit mapping gives statuses equal to the group mapping's.
    bc::Result rc = bc::fit_batch<bc::PseudoVoigt>(batch, opts, bc::KernelVariant::CtaPerFit);
    CHECK(rc.timings.variant == bc::KernelVariant::CtaPerFit);
    std::size_t same = 0;
    for (std::size_t i = 0; i < n; ++i)
        same += rc.status[i] == bc::FitStatus(status[i]);
    CHECK(same >= n * 999 / 1000);
    return 0;
}

int main(int argc, char **argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    try {
        gpu ? gpu_mode() : cpu_mode();
    } catch (const std::exception &e) {
        std::printf("FAIL uncaught %s\n", e.what());
        return 1;
    }
    if (failures)
        return 1;
    std::printf("OK\n");
    return 0;
}
