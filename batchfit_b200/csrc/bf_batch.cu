// Mixed batches on a context: host planner, device arena, CUDA-graph replay and
// the lanes-per-fit autotuner (include/batchfit_cuda.h, "Mixed batches").
//
// Planner.  Every segment (one fit call) becomes one LM run, filed under the class
// (model, lanes per fit, octave of M when several fits share a warp), and, when it
// has no p0, one guess run under (model, guess lanes, register width).  Classes are
// ordered by their costliest fit (M x LM state size), largest first, and runs
// within a class by M, largest first: the persistent kernels then finish on the
// cheapest fits.  Few, large classes matter: warps of one SM that run different
// classes run different template instantiations, which thrashes the instruction
// cache.  The fixed mapping (the plain baseline) files every fit of a model under
// one 32-lane class and keeps the call order.
//
// Arena.  One device allocation holds the batch header, segments, classes, runs,
// work items, class counters and the guess buffers.  Its layout depends only on
// its capacities, so the kernel arguments (pointers into it) stay fixed until it
// grows; the pipeline (counter reset + four kernels) is captured once into a CUDA
// graph and replayed for every batch that fits.  A batch uploads its descriptors
// (a few hundred bytes per segment) from a pinned mirror before the replay.
#include "bf_batch.h"
#include "bf_context.h"
#include "bf_kernels.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace bf {
namespace host {

namespace {

int parameter_count(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }
int state_size(int model) {
    const int p = parameter_count(model);
    return 1 + p + p * (p + 1) / 2;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Device arena layout for the given capacities.
struct Layout {
    size_t header, segs, lm_classes, guess_classes, lm_runs, guess_runs, lm_items, guess_items, counters, guesses,
        total;
};

Layout layout_for(size_t segs, size_t items, size_t guess_floats) {
    Layout l{};
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at = align_up(at + bytes, 256);
        return here;
    };
    l.header = take(sizeof(BatchHeader));
    l.segs = take(segs * sizeof(Segment));
    l.lm_classes = take(kMaxClasses * sizeof(WorkClass));
    l.guess_classes = take(kMaxClasses * sizeof(WorkClass));
    l.lm_runs = take(segs * sizeof(WorkRun));
    l.guess_runs = take(segs * sizeof(WorkRun));
    l.lm_items = take(items * sizeof(WorkItem));
    l.guess_items = take(items * sizeof(WorkItem));
    l.counters = take(2 * kMaxClasses * sizeof(unsigned long long));
    l.guesses = take(guess_floats * sizeof(float));
    l.total = at;
    return l;
}

int bucket_of(uint32_t m) {
    // Nearest of 64 * 2^b in log scale.
    const double b = std::log2(double(m < 1 ? 1 : m) / 64.0);
    const int r = int(std::lround(b));
    return r < 0 ? 0 : r > 7 ? 7 : r;
}

} // namespace

struct BatchState {
    DeviceBuffer arena;
    size_t seg_cap = 0, item_cap = 0, guess_cap = 0;
    Layout lay{};
    void *host = nullptr; // pinned mirror of header .. guess runs
    size_t host_bytes = 0;
    BatchArgs args{};
    cudaGraphExec_t graph = nullptr;
    cudaGraph_t graph_src = nullptr;               // the captured graph: its nodes address `graph`'s
    cudaGraphNode_t lm_nodes[kLmClassTypes] = {};  // LM kernel node per work-class type
    uint32_t lm_enabled = kAllLmTypes;             // LM nodes enabled in `graph`
    uint32_t kernels = 0;                          // kernels of the last direct launch
    LmFork fork;                                   // side streams of the LM kernels
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bf_tuning tuning{};
    bool warmed = false; // kernels' attributes set (before any capture)
};

void release_batch_state(BatchState *st) {
    if (!st)
        return;
    if (st->graph)
        cudaGraphExecDestroy(st->graph);
    if (st->graph_src)
        cudaGraphDestroy(st->graph_src);
    release_lm_fork(st->fork);
    st->arena.release();
    if (st->host)
        cudaFreeHost(st->host);
    for (cudaEvent_t e : st->ev)
        if (e)
            cudaEventDestroy(e);
    delete st;
}

namespace {

// Built-in lanes per fit before tuning: the single-batch path's choice.
void default_tuning(bf_tuning &t) {
    std::memset(&t, 0, sizeof(t));
    for (int model = 0; model < 4; ++model)
        for (int b = 0; b < 8; ++b)
            t.lanes[model][b] = default_lanes(model, uint32_t(64u << b));
}

int state_of(bf_cuda_context *ctx, BatchState **out) {
    if (!ctx->batch) {
        const int rc = create_batch_state(&ctx->batch);
        if (rc != BF_OK)
            return rc;
    }
    *out = ctx->batch;
    return BF_OK;
}

void drop_graph(BatchState &st) {
    if (st.graph)
        cudaGraphExecDestroy(st.graph);
    if (st.graph_src)
        cudaGraphDestroy(st.graph_src);
    st.graph = nullptr;
    st.graph_src = nullptr;
    std::fill(std::begin(st.lm_nodes), std::end(st.lm_nodes), nullptr);
    st.lm_enabled = kAllLmTypes;
}

// Capture the pipeline (every LM kernel) on `stream` and instantiate it; keep the
// captured graph and its LM kernel nodes, which batches enable per work-class type.
cudaError_t capture_graph(BatchState &st, int sms, cudaStream_t stream) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const cudaError_t le = launch_batch_pipeline(st.args, sms, stream, nullptr, nullptr, &st.fork);
        e = cudaStreamEndCapture(stream, &g);
        if (le != cudaSuccess)
            e = le;
    }
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&st.graph, g, 0);
    if (e != cudaSuccess) {
        if (g)
            cudaGraphDestroy(g);
        return e;
    }
    st.graph_src = g;
    st.lm_enabled = kAllLmTypes;
    size_t count = 0;
    e = cudaGraphGetNodes(g, nullptr, &count);
    std::vector<cudaGraphNode_t> nodes(count);
    if (e == cudaSuccess && count)
        e = cudaGraphGetNodes(g, nodes.data(), &count);
    for (size_t i = 0; i < count && e == cudaSuccess; ++i) {
        cudaGraphNodeType type;
        e = cudaGraphNodeGetType(nodes[i], &type);
        if (e != cudaSuccess || type != cudaGraphNodeTypeKernel)
            continue;
        cudaKernelNodeParams kp{};
        e = cudaGraphKernelNodeGetParams(nodes[i], &kp);
        for (int k = 0; k < kLmClassTypes && e == cudaSuccess; ++k)
            if (kp.func == batch_lm_function(k))
                st.lm_nodes[k] = nodes[i];
    }
    return e;
}

// Grow the arena (and drop the graph, whose arguments point into it).
int reserve(BatchState &st, size_t segs, size_t items, size_t guess_floats) {
    if (segs <= st.seg_cap && items <= st.item_cap && guess_floats <= st.guess_cap && st.arena.ptr)
        return BF_OK;
    const size_t s = std::max(segs + segs / 2, std::max<size_t>(st.seg_cap, 64));
    const size_t i = std::max(items + items / 4, std::max<size_t>(st.item_cap, 1024));
    const size_t g = std::max(guess_floats + guess_floats / 4, std::max<size_t>(st.guess_cap, 4096));
    const Layout lay = layout_for(s, i, g);
    drop_graph(st);
    st.arena.release();
    cudaError_t e = st.arena.reserve(lay.total);
    if (e != cudaSuccess)
        return report_cuda(e, "batch arena");
    const size_t host_bytes = lay.lm_items; // header .. guess runs
    if (host_bytes > st.host_bytes) {
        if (st.host)
            cudaFreeHost(st.host);
        st.host = nullptr;
        st.host_bytes = 0;
        e = cudaMallocHost(&st.host, host_bytes);
        if (e != cudaSuccess)
            return report_cuda(e, "batch descriptor mirror");
        st.host_bytes = host_bytes;
    }
    st.seg_cap = s;
    st.item_cap = i;
    st.guess_cap = g;
    st.lay = lay;
    char *base = static_cast<char *>(st.arena.ptr);
    st.args.hdr = reinterpret_cast<const BatchHeader *>(base + lay.header);
    st.args.segs = reinterpret_cast<Segment *>(base + lay.segs);
    st.args.lm_classes = reinterpret_cast<const WorkClass *>(base + lay.lm_classes);
    st.args.guess_classes = reinterpret_cast<const WorkClass *>(base + lay.guess_classes);
    st.args.lm_runs = reinterpret_cast<const WorkRun *>(base + lay.lm_runs);
    st.args.guess_runs = reinterpret_cast<const WorkRun *>(base + lay.guess_runs);
    st.args.lm_items = reinterpret_cast<WorkItem *>(base + lay.lm_items);
    st.args.guess_items = reinterpret_cast<WorkItem *>(base + lay.guess_items);
    st.args.counters = reinterpret_cast<unsigned long long *>(base + lay.counters);
    return BF_OK;
}

struct Plan {
    BatchHeader hdr{};
    std::vector<Segment> segs;
    std::vector<WorkClass> lm_classes, guess_classes;
    std::vector<WorkRun> lm_runs, guess_runs;
    size_t guess_floats = 0;
    bool any_guess = false, any_uncertain = false;
};

// Order runs into classes and assign item ranges.  `keys[r]` is the class key of
// run r, `cost[r]` its per-fit cost, `m[r]` its M.
using ClassKey = std::tuple<int, int, int, int>; // model, lanes, guess width, log2(M)

void order_runs(std::vector<WorkRun> &runs, const std::vector<ClassKey> &keys,
                const std::vector<double> &cost, const std::vector<uint32_t> &m, bool fixed,
                std::vector<WorkClass> &classes) {
    std::map<ClassKey, int> index;
    std::vector<std::vector<int>> members;
    std::vector<double> top;
    for (size_t r = 0; r < runs.size(); ++r) {
        auto it = index.find(keys[r]);
        if (it == index.end()) {
            it = index.emplace(keys[r], int(members.size())).first;
            members.emplace_back();
            top.push_back(0.0);
        }
        members[it->second].push_back(int(r));
        top[it->second] = std::max(top[it->second], cost[r]);
    }
    std::vector<int> order(members.size());
    for (size_t c = 0; c < order.size(); ++c)
        order[c] = int(c);
    if (!fixed)
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return top[a] > top[b]; });
    std::vector<ClassKey> key_of(members.size());
    for (auto &kv : index)
        key_of[kv.second] = kv.first;
    std::vector<WorkRun> sorted;
    sorted.reserve(runs.size());
    long long start = 0;
    for (int c : order) {
        auto &mem = members[c];
        if (!fixed)
            std::stable_sort(mem.begin(), mem.end(), [&](int a, int b) { return m[a] > m[b]; });
        WorkClass cls{};
        cls.model = std::get<0>(key_of[c]);
        cls.lanes = std::get<1>(key_of[c]);
        cls.v = std::get<2>(key_of[c]);
        cls.begin = start;
        for (int r : mem) {
            WorkRun run = runs[r];
            run.start = start;
            start += run.count;
            sorted.push_back(run);
        }
        cls.fits = start - cls.begin;
        classes.push_back(cls);
    }
    runs.swap(sorted);
}

int plan_batch(BatchState &st, const bf_batch_segment *segments, uint32_t count, uint32_t flags, int sms,
               Plan &plan) {
    const bool fixed = (flags & BF_BATCH_FIXED_MAPPING) != 0;
    std::vector<ClassKey> lm_keys, guess_keys;
    std::vector<char> tuned_width; // the run's lanes came from the tuning table
    std::vector<double> lm_cost, guess_cost;
    std::vector<uint32_t> lm_m, guess_m;
    size_t items = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const bf_fit_args &args = segments[i].args;
        FitArgs base{};
        int rc = prepare_segment(&args, &segments[i].out, uint32_t(kBatchMaxPoints), &base);
        if (rc != BF_OK)
            return report(rc, "segment " + std::to_string(i) + ": " + bf_cuda_last_error());
        if (args.memory != BF_MEMORY_DEVICE)
            return report(BF_ERR_INVALID_ARGUMENT,
                          "segment " + std::to_string(i) + ": mixed batches take device memory only");
        if (args.n > uint64_t(0x7fffffff))
            return report(BF_ERR_INVALID_ARGUMENT, "segment " + std::to_string(i) + ": more than 2^31-1 fits");
        if (args.n == 0)
            continue;
        const int p = parameter_count(args.model);
        Segment seg{};
        seg.a = base;
        seg.a.x = args.x;
        seg.a.y = args.y;
        seg.a.p0 = args.p0;
        seg.a.params = segments[i].out.params;
        seg.a.status = segments[i].out.status;
        seg.a.iterations = segments[i].out.iterations;
        seg.a.chi2 = segments[i].out.chi2;
        seg.a.covariance = segments[i].out.covariance;
        seg.a.stderr_out = segments[i].out.standard_errors;
        seg.a.ustatus = segments[i].out.uncertainty_status;
        seg.a.n = (long long)args.n;
        seg.a.work_counter = nullptr;
        seg.model = args.model;
        const int s = int(plan.segs.size());
        int lanes = args.group_lanes;
        tuned_width.push_back(lanes == 0 && !fixed);
        if (lanes == 0)
            lanes = fixed ? 32 : st.tuning.lanes[args.model][bucket_of(args.m)];
        // Fits of one class share a warp's code path; a class of several fits per warp
        // spans M within a factor of two, so that its groups run passes of similar
        // length.
        const int octave = fixed ? 0 : 31 - __builtin_clz(args.m);
        lm_keys.emplace_back(args.model, lanes, 0, octave);
        lm_cost.push_back(double(args.m) * state_size(args.model));
        lm_m.push_back(args.m);
        plan.lm_runs.push_back(WorkRun{s, 0, 0, (long long)args.n, 0});
        if (!args.p0) {
            int gl = 0, gv = 0;
            batch_guess_shape(int(args.m), &gl, &gv);
            // The shape bounds M to a factor of four within a guess class.
            guess_keys.emplace_back(args.model, gl, gv, 0);
            guess_cost.push_back(double(args.m));
            guess_m.push_back(args.m);
            plan.guess_runs.push_back(WorkRun{s, 0, 0, (long long)args.n, 0});
            seg.guesses = reinterpret_cast<float *>(plan.guess_floats); // offset, resolved below
            plan.guess_floats += align_up(size_t(args.n) * p, 64);
            plan.any_guess = true;
        }
        plan.any_uncertain = plan.any_uncertain || args.uncertainties;
        plan.hdr.uncertain_segments += args.uncertainties ? 1 : 0;
        items += size_t(args.n);
        plan.segs.push_back(seg);
    }
    // A class too small to fill the GPU a few times over is bound by the latency of
    // its slowest fits, not by throughput: its fits take whole warps (32 lanes), which
    // shortens every LM round.  The tuned narrower widths pay off for large classes.
    {
        std::map<ClassKey, long long> fits;
        for (size_t r = 0; r < lm_keys.size(); ++r)
            fits[lm_keys[r]] += plan.lm_runs[r].count;
        for (size_t r = 0; r < lm_keys.size(); ++r) {
            const int lanes = std::get<1>(lm_keys[r]);
            const long long slots = (long long)sms * 2 * (256 / lanes);
            if (tuned_width[r] && lanes < 32 && fits[lm_keys[r]] < 4 * slots)
                std::get<1>(lm_keys[r]) = 32;
        }
        // One fit per warp needs no split by M: 32-lane classes merge per model.
        for (auto &k : lm_keys)
            if (std::get<1>(k) == 32)
                std::get<3>(k) = 0;
    }
    order_runs(plan.lm_runs, lm_keys, lm_cost, lm_m, fixed, plan.lm_classes);
    order_runs(plan.guess_runs, guess_keys, guess_cost, guess_m, fixed, plan.guess_classes);
    if (plan.lm_classes.size() > size_t(kMaxClasses) || plan.guess_classes.size() > size_t(kMaxClasses))
        return report(BF_ERR_INVALID_ARGUMENT, "too many work classes");
    plan.hdr.segments = int(plan.segs.size());
    plan.hdr.lm_classes = int(plan.lm_classes.size());
    plan.hdr.guess_classes = int(plan.guess_classes.size());
    plan.hdr.lm_runs = int(plan.lm_runs.size());
    plan.hdr.guess_runs = int(plan.guess_runs.size());
    plan.hdr.lm_items = (long long)items;
    long long gi = 0;
    for (const WorkRun &r : plan.guess_runs)
        gi += r.count;
    plan.hdr.guess_items = gi;
    return BF_OK;
}

// Upload the plan's descriptors into the arena on `stream` (from the pinned mirror).
cudaError_t upload(BatchState &st, Plan &plan, cudaStream_t stream) {
    float *guess_base = reinterpret_cast<float *>(static_cast<char *>(st.arena.ptr) + st.lay.guesses);
    for (Segment &s : plan.segs) {
        if (s.a.p0 == nullptr) {
            s.guesses = guess_base + reinterpret_cast<size_t>(s.guesses);
            s.a.p0 = s.guesses;
        } else {
            s.guesses = nullptr;
        }
    }
    char *h = static_cast<char *>(st.host);
    std::memcpy(h + st.lay.header, &plan.hdr, sizeof(BatchHeader));
    std::memcpy(h + st.lay.segs, plan.segs.data(), plan.segs.size() * sizeof(Segment));
    std::memcpy(h + st.lay.lm_classes, plan.lm_classes.data(), plan.lm_classes.size() * sizeof(WorkClass));
    std::memcpy(h + st.lay.guess_classes, plan.guess_classes.data(), plan.guess_classes.size() * sizeof(WorkClass));
    std::memcpy(h + st.lay.lm_runs, plan.lm_runs.data(), plan.lm_runs.size() * sizeof(WorkRun));
    std::memcpy(h + st.lay.guess_runs, plan.guess_runs.data(), plan.guess_runs.size() * sizeof(WorkRun));
    char *d = static_cast<char *>(st.arena.ptr);
    auto put = [&](size_t off, size_t bytes) {
        return bytes ? cudaMemcpyAsync(d + off, h + off, bytes, cudaMemcpyHostToDevice, stream) : cudaSuccess;
    };
    // Header and class tables are contiguous; segments and runs are copied as used.
    cudaError_t e = put(st.lay.header, sizeof(BatchHeader));
    if (e == cudaSuccess)
        e = put(st.lay.segs, plan.segs.size() * sizeof(Segment));
    if (e == cudaSuccess)
        e = put(st.lay.lm_classes, st.lay.lm_runs - st.lay.lm_classes);
    if (e == cudaSuccess)
        e = put(st.lay.lm_runs, plan.lm_runs.size() * sizeof(WorkRun));
    if (e == cudaSuccess)
        e = put(st.lay.guess_runs, plan.guess_runs.size() * sizeof(WorkRun));
    return e;
}

} // namespace

// LM work-class types present in a plan (bit per type).
uint32_t lm_types_of(const Plan &plan) {
    uint32_t types = 0;
    for (const WorkClass &c : plan.lm_classes)
        types |= 1u << lm_class_type(c.model, c.lanes);
    return types;
}

// Plan, upload and launch one batch on `stream` with the arena and graph of `st`
// (events st.ev[0..3] bracket it).  Returns without waiting; *launched is false
// when the batch had no fits.  One batch per state may be in flight: the pinned
// descriptor mirror is reused by the next call.
int launch_planned(BatchState &st, const bf_batch_segment *segments, uint32_t count, uint32_t flags, int sms,
                   cudaStream_t stream, bool *launched, bool *graph_used) {
    *launched = false;
    *graph_used = false;
    Plan plan;
    int rc = plan_batch(st, segments, count, flags, sms, plan);
    if (rc != BF_OK)
        return rc;
    if (plan.segs.empty())
        return BF_OK;
    rc = reserve(st, plan.segs.size(), size_t(plan.hdr.lm_items), plan.guess_floats);
    if (rc != BF_OK)
        return rc;
    cudaError_t e = upload(st, plan, stream);
    if (e != cudaSuccess)
        return report_cuda(e, "batch descriptors");
    // Graph replay saves the host ~15 launches: it matters for short batches.  Large
    // batches launch directly: measured on B200 (mixed stream, 65,536 fits), the
    // LM kernels' three streams overlap their tails in direct launches (pipeline
    // 4.38 ms) but not in the replayed graph (4.67 ms).
    constexpr long long kGraphMaxItems = 32768;
    const bool use_graph = (flags & BF_BATCH_NO_GRAPH) == 0 && st.warmed && plan.hdr.lm_items < kGraphMaxItems;
    e = cudaEventRecord(st.ev[0], stream);
    const uint32_t types = lm_types_of(plan);
    if (e == cudaSuccess && use_graph) {
        if (!st.graph)
            e = capture_graph(st, sms, stream);
        // Only the LM kernels of the batch's work-class types run.
        for (int k = 0; k < kLmClassTypes && e == cudaSuccess; ++k) {
            const bool want = (types >> k & 1u) != 0;
            if (st.lm_nodes[k] && want != ((st.lm_enabled >> k & 1u) != 0)) {
                e = cudaGraphNodeSetEnabled(st.graph, st.lm_nodes[k], want ? 1u : 0u);
                st.lm_enabled ^= 1u << k;
            }
        }
        if (e == cudaSuccess)
            e = cudaGraphLaunch(st.graph, stream);
    } else if (e == cudaSuccess) {
        e = launch_batch_pipeline(st.args, sms, stream, st.ev[1], st.ev[2], &st.fork, types);
        st.warmed = st.warmed || e == cudaSuccess;
        st.kernels = 3u + uint32_t(__builtin_popcount(types)); // prepare, guess, LM per type, covariance
    }
    if (e == cudaSuccess)
        e = cudaEventRecord(st.ev[3], stream);
    if (e != cudaSuccess)
        return report_cuda(e, "mixed batch launch");
    *launched = true;
    *graph_used = use_graph;
    return BF_OK;
}

// Wait for the batch launched on `st` and report its device time.
int finish_planned(BatchState &st, bool graph_used, bf_cuda_timing *out) {
    cudaError_t e = cudaEventSynchronize(st.ev[3]);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess)
        return report_cuda(e, "mixed batch");
    float total = 0.0f;
    cudaEventElapsedTime(&total, st.ev[0], st.ev[3]);
    bf_cuda_timing t{};
    t.kernel_ms = total;
    t.total_ms = total;
    t.launches = graph_used ? 1u : st.kernels;
    t.batches = 1;
    if (!graph_used) {
        float g = 0.0f, l = 0.0f, c = 0.0f;
        cudaEventElapsedTime(&g, st.ev[0], st.ev[1]);
        cudaEventElapsedTime(&l, st.ev[1], st.ev[2]);
        cudaEventElapsedTime(&c, st.ev[2], st.ev[3]);
        t.guess_ms = g;
        t.lm_ms = l;
        t.covariance_ms = c;
    }
    if (out)
        *out = t;
    return BF_OK;
}

// Size the arena for `segs` segments and `fits` fits, set the kernels up and
// capture the graph, so that batches within those sizes neither allocate nor
// synchronise the device.
int prepare_planned(BatchState &st, size_t segs, size_t fits, int sms, cudaStream_t stream) {
    int rc = reserve(st, segs, fits, fits * 8);
    if (rc != BF_OK)
        return rc;
    BatchHeader empty{};
    std::memcpy(static_cast<char *>(st.host) + st.lay.header, &empty, sizeof(empty));
    cudaError_t e = cudaMemcpyAsync(static_cast<char *>(st.arena.ptr) + st.lay.header,
                                    static_cast<char *>(st.host) + st.lay.header, sizeof(empty),
                                    cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = launch_batch_pipeline(st.args, sms, stream, nullptr, nullptr, &st.fork);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return report_cuda(e, "batch warm-up");
    st.warmed = true;
    if (!st.graph) {
        e = capture_graph(st, sms, stream);
        if (e != cudaSuccess)
            return report_cuda(e, "batch graph");
    }
    return BF_OK;
}

bool planned_done(BatchState &st, cudaError_t *error) {
    const cudaError_t e = cudaEventQuery(st.ev[3]);
    *error = e == cudaErrorNotReady ? cudaSuccess : e;
    return e != cudaErrorNotReady;
}

int create_batch_state(BatchState **out) {
    auto *st = new BatchState();
    default_tuning(st->tuning);
    if (const cudaError_t err = create_lm_fork(st->fork); err != cudaSuccess) {
        release_batch_state(st);
        return report_cuda(err, "batch streams");
    }
    for (cudaEvent_t &e : st->ev) {
        const cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) {
            release_batch_state(st);
            return report_cuda(err, "batch events");
        }
    }
    *out = st;
    return BF_OK;
}

// Run one batch on the context's first stream and wait for it.
int run_batch(bf_cuda_context *ctx, const bf_batch_segment *segments, uint32_t count, uint32_t flags) {
    BatchState *st = nullptr;
    int rc = state_of(ctx, &st);
    if (rc != BF_OK)
        return rc;
    ctx->last = bf_cuda_timing{};
    bool launched = false, graph_used = false;
    rc = launch_planned(*st, segments, count, flags, ctx->sms, ctx->stream[0], &launched, &graph_used);
    if (rc != BF_OK || !launched)
        return rc;
    return finish_planned(*st, graph_used, &ctx->last);
}

bf_tuning &tuning_of(BatchState *st) { return st->tuning; }

int batch_state(bf_cuda_context *ctx, BatchState **out) { return state_of(ctx, out); }

} // namespace host
} // namespace bf

// ------------------------------------------------------------------ C ABI --
namespace {

using bf::host::report;
using bf::host::report_cuda;

// Holds the context for one call (the same exclusion as bf_cuda_submit).
struct ContextLease {
    bf_cuda_context *ctx;
    bool held = false;
    explicit ContextLease(bf_cuda_context *c) : ctx(c) { held = !ctx->busy.exchange(true); }
    ~ContextLease() {
        if (held)
            ctx->busy.store(false);
    }
};

// Lanes per fit for every (model, bucket): the LM kernel timed at 8, 16 and 32
// lanes on seeded synthetic spectra, fastest kept.
int autotune(bf_cuda_context *ctx, bf_tuning *out) {
    bf::host::BatchState *st = nullptr;
    int rc = bf::host::batch_state(ctx, &st);
    if (rc != BF_OK)
        return rc;
    const long long min_fits = 4ll * ctx->sms * 64; // four waves of 8-lane groups
    long long max_points = 0, max_fits = 0;
    for (int b = 0; b < 8; ++b) {
        const long long m = 64ll << b;
        const long long n = std::max(min_fits, (1ll << 24) / m);
        max_points = std::max(max_points, n * m);
        max_fits = std::max(max_fits, n);
    }
    bf::host::DeviceBuffer x, y, params, status, iters, chi2;
    cudaError_t e = x.reserve(sizeof(float) * (64 << 7));
    if (e == cudaSuccess)
        e = y.reserve(sizeof(float) * size_t(max_points));
    if (e == cudaSuccess)
        e = params.reserve(sizeof(float) * 8 * size_t(max_fits));
    if (e == cudaSuccess)
        e = status.reserve(sizeof(int32_t) * size_t(max_fits));
    if (e == cudaSuccess)
        e = iters.reserve(sizeof(uint32_t) * size_t(max_fits));
    if (e == cudaSuccess)
        e = chi2.reserve(sizeof(float) * size_t(max_fits));
    bf_tuning t{};
    for (int model = 0; model < 4 && e == cudaSuccess && rc == BF_OK; ++model) {
        for (int b = 0; b < 8 && e == cudaSuccess && rc == BF_OK; ++b) {
            const int m = 64 << b;
            const long long n = std::max(min_fits, (1ll << 24) / m);
            e = bf::launch_synthetic(model, m, n, 0x5eed0000u + 64u * unsigned(model) + unsigned(b),
                                     static_cast<float *>(x.ptr), static_cast<float *>(y.ptr), ctx->stream[0]);
            if (e != cudaSuccess)
                break;
            bf_batch_segment seg{};
            seg.args.model = model;
            seg.args.n = uint64_t(n);
            seg.args.m = uint32_t(m);
            seg.args.x = static_cast<const float *>(x.ptr);
            seg.args.y = static_cast<const float *>(y.ptr);
            seg.args.memory = BF_MEMORY_DEVICE;
            bf_cuda_default_options(model, BF_POLICY_PARITY, &seg.args.options);
            seg.out.params = static_cast<float *>(params.ptr);
            seg.out.status = static_cast<int32_t *>(status.ptr);
            seg.out.iterations = static_cast<uint32_t *>(iters.ptr);
            seg.out.chi2 = static_cast<float *>(chi2.ptr);
            double best = 0.0;
            int best_lanes = 8;
            const int widths[3] = {8, 16, 32};
            for (int w = 0; w < 3 && rc == BF_OK; ++w) {
                seg.args.group_lanes = widths[w];
                double fastest = 0.0;
                for (int rep = 0; rep < 2 && rc == BF_OK; ++rep) {
                    rc = bf::host::run_batch(ctx, &seg, 1, BF_BATCH_NO_GRAPH);
                    const double ms = ctx->last.lm_ms;
                    fastest = rep == 0 ? ms : std::min(fastest, ms);
                }
                t.lm_ms[model][b][w] = fastest;
                if (w == 0 || fastest < best) {
                    best = fastest;
                    best_lanes = widths[w];
                }
            }
            t.lanes[model][b] = best_lanes;
        }
    }
    if (e != cudaSuccess)
        rc = report_cuda(e, "autotune");
    for (auto *buf : {&x, &y, &params, &status, &iters, &chi2})
        buf->release();
    ctx->last = bf_cuda_timing{};
    if (rc != BF_OK)
        return rc;
    t.tuned = 1;
    bf::host::tuning_of(st) = t;
    if (out)
        *out = t;
    return BF_OK;
}

} // namespace

extern "C" {

uint32_t bf_cuda_batch_max_points(void) { return uint32_t(bf::kBatchMaxPoints); }

int bf_cuda_fit_batch(bf_cuda_context *ctx, const bf_batch_segment *segments, uint32_t count, uint32_t flags) {
    if (!ctx || (count > 0 && !segments))
        return report(BF_ERR_INVALID_ARGUMENT, "null context or segment list");
    if (flags & ~(BF_BATCH_FIXED_MAPPING | BF_BATCH_NO_GRAPH))
        return report(BF_ERR_INVALID_ARGUMENT, "unknown batch flags");
    ContextLease lease(ctx);
    if (!lease.held)
        return report(BF_ERR_BUSY, "a submission is already in flight on this context");
    std::lock_guard<std::mutex> lock(ctx->mutex);
    const cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return report_cuda(e, "cudaSetDevice");
    return bf::host::run_batch(ctx, segments, count, flags);
}

int bf_cuda_autotune(bf_cuda_context *ctx, bf_tuning *out) {
    if (!ctx)
        return report(BF_ERR_INVALID_ARGUMENT, "null context");
    ContextLease lease(ctx);
    if (!lease.held)
        return report(BF_ERR_BUSY, "a submission is already in flight on this context");
    std::lock_guard<std::mutex> lock(ctx->mutex);
    const cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return report_cuda(e, "cudaSetDevice");
    return autotune(ctx, out);
}

int bf_cuda_get_tuning(bf_cuda_context *ctx, bf_tuning *out) {
    if (!ctx || !out)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(ctx->mutex);
    bf::host::BatchState *st = nullptr;
    const int rc = bf::host::batch_state(ctx, &st);
    if (rc == BF_OK)
        *out = bf::host::tuning_of(st);
    return rc;
}

int bf_cuda_set_tuning(bf_cuda_context *ctx, const bf_tuning *in) {
    if (!ctx || !in)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    for (int model = 0; model < 4; ++model)
        for (int b = 0; b < 8; ++b) {
            const int l = in->lanes[model][b];
            if (l != 8 && l != 16 && l != 32)
                return report(BF_ERR_INVALID_ARGUMENT, "tuning lanes must be 8, 16 or 32");
        }
    std::lock_guard<std::mutex> lock(ctx->mutex);
    bf::host::BatchState *st = nullptr;
    const int rc = bf::host::batch_state(ctx, &st);
    if (rc == BF_OK) {
        bf::host::tuning_of(st) = *in;
        bf::host::tuning_of(st).tuned = 1;
    }
    return rc;
}

} // extern "C"
