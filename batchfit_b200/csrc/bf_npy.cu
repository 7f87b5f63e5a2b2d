// Out-of-core fitting from NPY files (include/batchfit_cuda.h, "NPY streaming").
//
// The reference streams fit-major y[N,M] from .npy files through its Metal batches
// (metal::fit_npy, include/batchfit/metal/pipeline.hpp:49-67; src/metal/pipeline.cpp:
// 70-265) and its tool writes parameters, chi-squared, status and iterations as
// .npy files (tools/fit_npy.cpp:20-121).  Here a reader thread fills pinned host
// chunks straight from the files (float64 inputs converted to float32 on the way)
// while the GPU fits the previous chunk through bf_cuda_fit's host path, which
// overlaps each chunk's copies with its kernels; results are appended to the
// output files in input order.  y stays fit-major: no transpose.
#include "batchfit_cuda.h"
#include "bf_context.h"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <fcntl.h>
#include <vector>

namespace {

using bf::host::report;

int parameters(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }

// ------------------------------------------------------------ NPY format --
// Little-endian float32 / float64 / uint32, C order, rank 1 or 2, format 1.0 or
// 2.0 -- the files numpy.save writes and the reference's reader accepts
// (src/cpu/npy.cpp:50-86).
struct Header {
    int dtype = -1; // 0 <f4, 1 <f8, 2 <u4
    int rank = 0;
    uint64_t shape[2] = {0, 0};
    size_t offset = 0;
    size_t item = 0;
};

bool skip_space(const std::string &t, size_t &i) {
    while (i < t.size() && (t[i] == ' ' || t[i] == '\t'))
        ++i;
    return i < t.size();
}

// Value text of `key` in the header dictionary.
bool field(const std::string &t, const char *key, size_t &at) {
    for (const char q : {'\'', '"'}) {
        const std::string k = std::string(1, q) + key + q;
        const size_t p = t.find(k);
        if (p == std::string::npos)
            continue;
        size_t i = p + k.size();
        if (!skip_space(t, i) || t[i] != ':')
            return false;
        ++i;
        if (!skip_space(t, i))
            return false;
        at = i;
        return true;
    }
    return false;
}

int read_header(const char *path, Header &h, std::string &why) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        why = std::string("cannot open ") + path + ": " + std::strerror(errno);
        return BF_ERR_INVALID_ARGUMENT;
    }
    unsigned char pre[12] = {};
    const size_t got = std::fread(pre, 1, 10, f);
    int rc = BF_OK;
    std::string text;
    size_t len = 0, start = 10;
    if (got != 10 || std::memcmp(pre, "\x93NUMPY", 6) != 0 || (pre[6] != 1 && pre[6] != 2)) {
        why = std::string(path) + ": not an NPY format 1.0/2.0 file";
        rc = BF_ERR_INVALID_ARGUMENT;
    } else if (pre[6] == 1) {
        len = size_t(pre[8]) | (size_t(pre[9]) << 8);
    } else if (std::fread(pre + 10, 1, 2, f) == 2) {
        len = size_t(pre[8]) | (size_t(pre[9]) << 8) | (size_t(pre[10]) << 16) | (size_t(pre[11]) << 24);
        start = 12;
    } else {
        why = std::string(path) + ": truncated header";
        rc = BF_ERR_INVALID_ARGUMENT;
    }
    if (rc == BF_OK && (len == 0 || len > (1u << 20))) {
        why = std::string(path) + ": invalid header length";
        rc = BF_ERR_INVALID_ARGUMENT;
    }
    if (rc == BF_OK) {
        text.resize(len);
        if (std::fread(&text[0], 1, len, f) != len) {
            why = std::string(path) + ": truncated header";
            rc = BF_ERR_INVALID_ARGUMENT;
        }
    }
    long long file_size = -1;
    if (rc == BF_OK && std::fseek(f, 0, SEEK_END) == 0)
        file_size = std::ftell(f);
    std::fclose(f);
    if (rc != BF_OK)
        return rc;
    size_t i = 0;
    auto bad = [&](const char *what) {
        why = std::string(path) + ": unsupported header (" + what + "; requires <f4/<f8/<u4, C order, rank 1/2)";
        return BF_ERR_INVALID_ARGUMENT;
    };
    if (!field(text, "descr", i))
        return bad("no descr");
    const std::string d = text.substr(i, 5);
    if (d == "'<f4'" || d == "\"<f4\"")
        h.dtype = 0;
    else if (d == "'<f8'" || d == "\"<f8\"")
        h.dtype = 1;
    else if (d == "'<u4'" || d == "\"<u4\"")
        h.dtype = 2;
    else
        return bad("dtype");
    h.item = h.dtype == 1 ? 8 : 4;
    if (!field(text, "fortran_order", i) || text.compare(i, 5, "False") != 0)
        return bad("fortran order");
    if (!field(text, "shape", i) || text[i] != '(')
        return bad("shape");
    ++i;
    h.rank = 0;
    while (true) {
        if (!skip_space(text, i))
            return bad("shape");
        if (text[i] == ')')
            break;
        if (text[i] < '0' || text[i] > '9' || h.rank == 2)
            return bad("shape");
        uint64_t v = 0;
        while (i < text.size() && text[i] >= '0' && text[i] <= '9') {
            if (v > (~0ull) / 10 - 10)
                return bad("shape");
            v = v * 10 + uint64_t(text[i] - '0');
            ++i;
        }
        h.shape[h.rank++] = v;
        if (!skip_space(text, i))
            return bad("shape");
        if (text[i] == ',')
            ++i;
    }
    if (h.rank < 1)
        return bad("rank 0");
    h.offset = start + len;
    uint64_t elements = h.shape[0] * (h.rank == 2 ? h.shape[1] : 1);
    if (file_size < 0 || uint64_t(file_size) != h.offset + elements * h.item) {
        why = std::string(path) + ": payload length does not match shape";
        return BF_ERR_INVALID_ARGUMENT;
    }
    return BF_OK;
}

// Format-1.0 writer whose shape is known up front (the reference's npy::Writer,
// src/cpu/npy.cpp:93-130): 64-byte aligned header, then appended rows.
struct Writer {
    FILE *f = nullptr;
    std::string path;
    uint64_t remaining = 0;
    size_t item = 4;
    int open(const std::string &p, const std::vector<uint64_t> &shape, const char *descr, std::string &why) {
        path = p;
        remaining = 1;
        std::string dims;
        for (uint64_t d : shape) {
            remaining *= d;
            dims += std::to_string(d) + ", ";
        }
        if (shape.size() > 1)
            dims.resize(dims.size() - 2);
        else
            dims.resize(dims.size() - 1);
        std::string hdr = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (" + dims +
                          "), }";
        hdr.append((64 - (10 + hdr.size() + 1) % 64) % 64, ' ');
        hdr += '\n';
        f = std::fopen(p.c_str(), "wb");
        if (!f) {
            why = "cannot create " + p + ": " + std::strerror(errno);
            return BF_ERR_INVALID_ARGUMENT;
        }
        const unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(hdr.size() & 255),
                                       (unsigned char)(hdr.size() >> 8)};
        if (std::fwrite(pre, 1, 10, f) != 10 || std::fwrite(hdr.data(), 1, hdr.size(), f) != hdr.size()) {
            why = "write failed: " + p;
            return BF_ERR_INVALID_ARGUMENT;
        }
        return BF_OK;
    }
    int append(const void *data, uint64_t count, std::string &why) {
        if (count > remaining || (count && std::fwrite(data, item, count, f) != count)) {
            why = "write failed: " + path;
            return BF_ERR_INVALID_ARGUMENT;
        }
        remaining -= count;
        return BF_OK;
    }
    int finish(std::string &why) {
        const bool ok = f && remaining == 0 && std::fclose(f) == 0;
        f = nullptr;
        if (!ok) {
            why = "incomplete output: " + path;
            return BF_ERR_INVALID_ARGUMENT;
        }
        return BF_OK;
    }
    ~Writer() {
        if (f)
            std::fclose(f);
    }
};

// Read `count` values starting at element `first` of an NPY payload as float32
// (float64 payloads go through `tmp` and are rounded to nearest).
bool read_floats(int fd, const Header &h, uint64_t first, uint64_t count, float *out, std::vector<double> &tmp) {
    char *dst = reinterpret_cast<char *>(out);
    if (h.dtype == 1) {
        tmp.resize(count);
        dst = reinterpret_cast<char *>(tmp.data());
    }
    const off_t off = off_t(h.offset + first * h.item);
    const size_t bytes = size_t(count * h.item);
    size_t done = 0;
    while (done < bytes) {
        const ssize_t r = pread(fd, dst + done, bytes - done, off + off_t(done));
        if (r <= 0)
            return false;
        done += size_t(r);
    }
    if (h.dtype == 1)
        for (uint64_t i = 0; i < count; ++i)
            out[i] = float(tmp[i]);
    return true;
}

struct Chunk {
    uint64_t first = 0, count = 0;
    float *y = nullptr, *p0 = nullptr;
    bool ready = false, failed = false;
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

} // namespace

extern "C" {

int bf_npy_inspect(const char *path, int32_t *dtype, int32_t *rank, uint64_t *shape) {
    if (!path || !dtype || !rank || !shape)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    Header h;
    std::string why;
    const int rc = read_header(path, h, why);
    if (rc != BF_OK)
        return report(rc, why);
    *dtype = h.dtype;
    *rank = h.rank;
    shape[0] = h.shape[0];
    shape[1] = h.rank == 2 ? h.shape[1] : 0;
    return BF_OK;
}

int bf_cuda_fit_npy(bf_cuda_context *ctx, const char *x_path, const char *y_path, const char *initial_path,
                    const char *output_dir, const bf_npy_options *options, bf_npy_stats *stats) {
    if (!ctx || !x_path || !y_path || !output_dir || !options)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    const double t_begin = now_s();
    const int model = options->model;
    if (model < 0 || model > 3)
        return report(BF_ERR_INVALID_ARGUMENT, "unknown model id");
    if (options->in_flight > 3)
        return report(BF_ERR_INVALID_ARGUMENT, "in_flight must be 1..3 (0 = 3)");
    const int p = parameters(model);
    Header hx, hy, hp;
    std::string why;
    int rc = read_header(x_path, hx, why);
    if (rc == BF_OK)
        rc = read_header(y_path, hy, why);
    if (rc == BF_OK && initial_path)
        rc = read_header(initial_path, hp, why);
    if (rc != BF_OK)
        return report(rc, why);
    if (hx.rank != 1 || hx.dtype == 2)
        return report(BF_ERR_INVALID_ARGUMENT, "x must be a float32/float64 array of shape [M]");
    if (hy.rank != 2 || hy.dtype == 2 || hy.shape[1] != hx.shape[0])
        return report(BF_ERR_INVALID_ARGUMENT, "y must be a float32/float64 array of shape [N,M] matching x[M]");
    if (initial_path && (hp.rank != 2 || hp.dtype == 2 || hp.shape[0] != hy.shape[0] || hp.shape[1] != uint64_t(p)))
        return report(BF_ERR_INVALID_ARGUMENT, "initial must be a float32/float64 array of shape [N,P]");
    const uint64_t n = hy.shape[0], m = hy.shape[1];
    if (m == 0 || m > 0xffffffffull)
        return report(BF_ERR_INVALID_ARGUMENT, "x must be nonempty");
    uint64_t chunk = options->chunk_fits;
    if (chunk == 0)
        chunk = std::max<uint64_t>(16384, (128ull << 20) / (m * 4));
    chunk = std::max<uint64_t>(1, std::min<uint64_t>(chunk, n ? n : 1));
    const unsigned slots = options->in_flight ? options->in_flight : 3;
    // The reference refuses an existing output directory (tools/fit_npy.cpp:28-29).
    if (mkdir(output_dir, 0777) != 0)
        return report(BF_ERR_INVALID_ARGUMENT, std::string("output directory must not already exist: ") + output_dir);
    const std::string dir(output_dir);
    std::vector<std::string> written;
    auto cleanup = [&]() {
        for (auto &f : written)
            std::remove(f.c_str());
        rmdir(output_dir);
    };

    // x, once.
    std::vector<float> x(m);
    std::vector<double> tmp;
    int fx = open(x_path, O_RDONLY), fy = open(y_path, O_RDONLY), fp = initial_path ? open(initial_path, O_RDONLY) : -1;
    bool ok = fx >= 0 && fy >= 0 && (!initial_path || fp >= 0) && read_floats(fx, hx, 0, m, x.data(), tmp);
    if (fx >= 0)
        close(fx);
    if (!ok) {
        if (fy >= 0)
            close(fy);
        if (fp >= 0)
            close(fp);
        cleanup();
        return report(BF_ERR_INVALID_ARGUMENT, "reading the input files failed");
    }

    // Output files (the reference tool's four, plus the uncertainty outputs).
    Writer w_par, w_chi, w_status, w_iter, w_cov, w_se, w_us;
    struct Out {
        Writer *w;
        const char *name;
        std::vector<uint64_t> shape;
        const char *descr;
    };
    const uint64_t pp = uint64_t(p);
    std::vector<Out> outs = {{&w_par, "parameters.npy", {n, pp}, "<f4"},
                             {&w_chi, "chi_squared.npy", {n}, "<f4"},
                             {&w_status, "status.npy", {n}, "<u4"},
                             {&w_iter, "iterations.npy", {n}, "<u4"}};
    if (options->uncertainties) {
        outs.push_back({&w_cov, "covariance.npy", {n, pp, pp}, "<f4"});
        outs.push_back({&w_se, "standard_errors.npy", {n, pp}, "<f4"});
        outs.push_back({&w_us, "uncertainty_status.npy", {n}, "<u4"});
    }
    for (auto &o : outs) {
        const std::string path = dir + "/" + o.name;
        rc = o.w->open(path, o.shape, o.descr, why);
        written.push_back(path);
        if (rc != BF_OK)
            break;
    }
    if (rc != BF_OK) {
        close(fy);
        if (fp >= 0)
            close(fp);
        cleanup();
        return report(rc, why);
    }

    // Pinned chunks: inputs and outputs of `slots` chunks.
    std::vector<Chunk> ring(slots);
    std::vector<void *> pinned;
    auto pin = [&](size_t bytes) -> void * {
        void *ptr = nullptr;
        if (bf_cuda_host_alloc(bytes ? bytes : 4, &ptr) != BF_OK)
            return nullptr;
        pinned.push_back(ptr);
        return ptr;
    };
    struct SlotOut {
        float *params, *chi2, *cov, *se;
        int32_t *status, *us;
        uint32_t *iters;
    };
    std::vector<SlotOut> sout(slots);
    for (unsigned s = 0; s < slots && ok; ++s) {
        ring[s].y = static_cast<float *>(pin(chunk * m * 4));
        ring[s].p0 = initial_path ? static_cast<float *>(pin(chunk * p * 4)) : nullptr;
        sout[s].params = static_cast<float *>(pin(chunk * p * 4));
        sout[s].chi2 = static_cast<float *>(pin(chunk * 4));
        sout[s].status = static_cast<int32_t *>(pin(chunk * 4));
        sout[s].iters = static_cast<uint32_t *>(pin(chunk * 4));
        sout[s].cov = options->uncertainties ? static_cast<float *>(pin(chunk * p * p * 4)) : nullptr;
        sout[s].se = options->uncertainties ? static_cast<float *>(pin(chunk * p * 4)) : nullptr;
        sout[s].us = options->uncertainties ? static_cast<int32_t *>(pin(chunk * 4)) : nullptr;
        ok = ring[s].y && sout[s].params && sout[s].chi2 && sout[s].status && sout[s].iters &&
             (!initial_path || ring[s].p0) && (!options->uncertainties || (sout[s].cov && sout[s].se && sout[s].us));
    }

    const uint64_t chunks = n ? (n + chunk - 1) / chunk : 0;
    std::mutex mutex;
    std::condition_variable cv;
    bool stop = false;
    double read_seconds = 0.0;
    std::vector<char> busy(slots, 0); // 1 while a chunk occupies the slot
    std::thread reader;
    if (ok) {
        reader = std::thread([&]() {
            std::vector<double> scratch;
            for (uint64_t c = 0; c < chunks; ++c) {
                const unsigned s = unsigned(c % slots);
                {
                    std::unique_lock<std::mutex> lock(mutex);
                    cv.wait(lock, [&] { return stop || !busy[s]; });
                    if (stop)
                        return;
                    busy[s] = 1;
                }
                const double t0 = now_s();
                Chunk &ch = ring[s];
                ch.first = c * chunk;
                ch.count = std::min(chunk, n - ch.first);
                bool good = read_floats(fy, hy, ch.first * m, ch.count * m, ch.y, scratch);
                if (good && initial_path)
                    good = read_floats(fp, hp, ch.first * p, ch.count * p, ch.p0, scratch);
                {
                    std::lock_guard<std::mutex> lock(mutex);
                    read_seconds += now_s() - t0;
                    ch.failed = !good;
                    ch.ready = true;
                }
                cv.notify_all();
            }
        });
    }

    double fit_seconds = 0.0, write_seconds = 0.0;
    for (uint64_t c = 0; c < chunks && ok; ++c) {
        const unsigned s = unsigned(c % slots);
        Chunk &ch = ring[s];
        {
            std::unique_lock<std::mutex> lock(mutex);
            cv.wait(lock, [&] { return ch.ready; });
            ch.ready = false;
        }
        if (ch.failed) {
            rc = BF_ERR_INVALID_ARGUMENT;
            why = "reading the input files failed";
            ok = false;
            break;
        }
        const double t0 = now_s();
        bf_fit_args args{};
        args.model = model;
        args.n = ch.count;
        args.m = uint32_t(m);
        args.x = x.data();
        args.y = ch.y;
        args.p0 = initial_path ? ch.p0 : nullptr;
        args.memory = BF_MEMORY_HOST;
        args.uncertainties = options->uncertainties ? 1 : 0;
        args.group_lanes = 0;
        args.options = options->solver;
        bf_fit_outputs out{sout[s].params, sout[s].status, sout[s].iters, sout[s].chi2,
                           sout[s].cov,    sout[s].se,     sout[s].us};
        rc = bf_cuda_fit(ctx, &args, &out);
        const double t1 = now_s();
        fit_seconds += t1 - t0;
        if (rc != BF_OK) {
            why = bf_cuda_last_error();
            ok = false;
            break;
        }
        // FitStatus codes are small non-negative integers: written as uint32
        // (tools/fit_npy.cpp:43-46).
        rc = w_par.append(sout[s].params, ch.count * p, why);
        if (rc == BF_OK)
            rc = w_chi.append(sout[s].chi2, ch.count, why);
        if (rc == BF_OK)
            rc = w_status.append(sout[s].status, ch.count, why);
        if (rc == BF_OK)
            rc = w_iter.append(sout[s].iters, ch.count, why);
        if (rc == BF_OK && options->uncertainties) {
            rc = w_cov.append(sout[s].cov, ch.count * p * p, why);
            if (rc == BF_OK)
                rc = w_se.append(sout[s].se, ch.count * p, why);
            if (rc == BF_OK)
                rc = w_us.append(sout[s].us, ch.count, why);
        }
        write_seconds += now_s() - t1;
        if (rc != BF_OK) {
            ok = false;
            break;
        }
        {
            std::lock_guard<std::mutex> lock(mutex);
            busy[s] = 0;
        }
        cv.notify_all();
    }
    {
        std::lock_guard<std::mutex> lock(mutex);
        stop = true;
    }
    cv.notify_all();
    if (reader.joinable())
        reader.join();
    close(fy);
    if (fp >= 0)
        close(fp);
    for (void *ptr : pinned)
        bf_cuda_host_free(ptr);
    if (ok) {
        for (auto &o : outs)
            if (rc == BF_OK)
                rc = o.w->finish(why);
        ok = rc == BF_OK;
    }
    if (!ok) {
        for (auto &o : outs)
            if (o.w->f) {
                std::fclose(o.w->f);
                o.w->f = nullptr;
            }
        cleanup();
        return report(rc != BF_OK ? rc : BF_ERR_INVALID_ARGUMENT, why.empty() ? "pinned host memory" : why);
    }
    if (stats) {
        stats->fits = n;
        stats->chunks = chunks;
        stats->chunk_fits = chunk;
        stats->wall_seconds = now_s() - t_begin;
        stats->read_seconds = read_seconds;
        stats->fit_seconds = fit_seconds;
        stats->write_seconds = write_seconds;
    }
    return BF_OK;
}

} // extern "C"
