/* batchfit_cuda.h -- C ABI of the batchfit B200 (sm_100a) fitting backend.
 *
 * A drop-in CUDA device for batchfit's fit path: shared x[M], fit-major y[N,M],
 * optional initial values p0[N,P] (NULL -> data-only guesses on the GPU), common
 * lower/upper bounds (equal bounds fix a coordinate), outputs params[N,P],
 * status/iterations/chi2[N] and optional covariance[N,P,P], stderr[N,P],
 * uncertainty_status[N].  Plain pointers and sizes only; no CUDA or framework types.
 *
 * Reference interfaces each entry point replaces (paths inside the batchfit project):
 *   bf_cuda_context_create/destroy  metal::Context (include/batchfit/metal/batch.hpp:160-174)
 *   bf_cuda_fit                     fit_batch<Model>(SharedBatch&, Device, options)
 *                                   (include/batchfit/metal/batch.hpp:268-310) and the Python
 *                                   native entry _core.fit (python/bindings.cpp:200-207)
 *   bf_cuda_submit / _ready / _wait submit_batch<Model> -> PendingBatch{ready(),get()}
 *                                   (include/batchfit/metal/batch.hpp:198-217,253-264)
 *   bf_cuda_guess                   cpu::initial_guess<float,Model> per row
 *                                   (include/batchfit/cpu/initial_guess.hpp:120-249)
 *   bf_solver_options               cpu::SolverOptions<float,P> (include/batchfit/cpu/solver.hpp:26-41)
 *   status / uncertainty codes      FitStatus (solver.hpp:16-23), UncertaintyStatus
 *                                   (include/batchfit/uncertainty_types.hpp:3-10)
 *   bf_cuda_available               batchfit.metal_available() (python/batchfit/__init__.py:51-53)
 *
 * Ownership: the caller owns every input and output buffer; the library owns its
 * device staging buffers, streams and events.  Threading: calls on one context are
 * serialised internally.  Per-fit failures are status codes, never error returns;
 * argument, device and CUDA failures return a nonzero code with a message from
 * bf_cuda_last_error() (thread-local).
 */
#ifndef BATCHFIT_CUDA_H
#define BATCHFIT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
#define BF_OK 0
#define BF_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define BF_ERR_CUDA 2             /* a CUDA runtime error (std::runtime_error) */
#define BF_ERR_UNAVAILABLE 3      /* no usable sm_100 device */
#define BF_ERR_BUSY 4             /* a pending submission still owns the context */
#define BF_ERR_CANCELLED 5        /* a server request cancelled before it was admitted */

/* Model ids (python/batchfit/__init__.py:13). */
#define BF_MODEL_GAUSSIAN 0       /* amplitude, center, sigma */
#define BF_MODEL_LORENTZIAN 1     /* amplitude, center, hwhm */
#define BF_MODEL_PSEUDO_VOIGT 2   /* amplitude, center, fwhm, mixing */
#define BF_MODEL_TWO_LORENTZIAN 3 /* a1, c1, hwhm1, a2, c2, hwhm2, intercept, slope */

/* Where the pointers of one call live. */
#define BF_MEMORY_HOST 0   /* host memory (pinned memory overlaps copies with compute) */
#define BF_MEMORY_DEVICE 1 /* device memory of the context's GPU */

/* Storage of y.  BF_Y_FLOAT16 is an opt-in half-precision storage, like the
 * reference's profiling variant (src/metal/profile_variants.metal:12-15): y holds
 * IEEE binary16 values, which halves y's host-to-device and HBM bytes; each value
 * is converted exactly to float32 on the GPU, so the fit equals the float32 fit of
 * the same (already rounded) values.  Accepted by bf_cuda_fit and bf_cuda_submit;
 * the other entry points take float32 y. */
#define BF_Y_FLOAT32 0
#define BF_Y_FLOAT16 1

/* Stopping policy.
 * BF_POLICY_REFERENCE: the reference float solver's stop rules with the given
 *   tolerances (defaults 1e-5 / 1e-6 / 1e-6).
 * BF_POLICY_PARITY: stop rules aimed at the float64 solution: the double-precision
 *   tolerances (1e-10 / 1e-10 / 1e-12) plus two float32 noise-floor tests -- every
 *   free |g_k| <= noise_floor * FLT_EPSILON * sqrt(A_kk * sum(y^2)), or an undamped
 *   step <= step_quantum * FLT_EPSILON * max|p|.  Statuses keep their meaning. */
#define BF_POLICY_REFERENCE 0
#define BF_POLICY_PARITY 1

typedef struct bf_solver_options {
    uint32_t max_iterations;   /* 100 */
    double initial_lambda;     /* 1e-3 */
    double gradient_tolerance; /* see BF_POLICY_* */
    double step_tolerance;
    double cost_tolerance;
    uint32_t compensated_sum; /* accepted for API parity: sums are always compensated */
    uint32_t scaled_cholesky; /* diagonal equilibration in the damped solve */
    uint32_t policy;          /* BF_POLICY_* */
    double noise_floor;       /* parity policy, multiples of FLT_EPSILON (16) */
    double step_quantum;      /* parity policy, multiples of FLT_EPSILON (16) */
    float lower[8];           /* per-parameter bounds, first P used; -inf/inf = unbounded */
    float upper[8];
} bf_solver_options;

typedef struct bf_fit_args {
    int32_t model;     /* BF_MODEL_* */
    uint64_t n;        /* fits */
    uint32_t m;        /* points per fit */
    const float *x;    /* [M] shared grid */
    const float *y;    /* [N*M] fit-major observations */
    const float *p0;   /* [N*P] initial values, or NULL for data-only guesses */
    int32_t memory;    /* BF_MEMORY_* for x, y, p0 and every output */
    int32_t uncertainties;
    int32_t group_lanes; /* 0 = tuned choice, else 8, 16 or 32 lanes per fit, or 128 = one CTA per fit */
    bf_solver_options options;
    int32_t y_format;    /* BF_Y_FLOAT32, or BF_Y_FLOAT16 (bf_cuda_fit / submit only) */
} bf_fit_args;

typedef struct bf_fit_outputs {
    float *params;              /* [N*P] */
    int32_t *status;            /* [N] FitStatus */
    uint32_t *iterations;       /* [N] */
    float *chi2;                /* [N] unweighted sum of squared residuals */
    float *covariance;          /* [N*P*P] when uncertainties */
    float *standard_errors;     /* [N*P] when uncertainties */
    int32_t *uncertainty_status;/* [N] when uncertainties */
} bf_fit_outputs;

typedef struct bf_cuda_context bf_cuda_context;
typedef struct bf_cuda_pending bf_cuda_pending;

/* Timing of the last completed call on a context (CUDA events, milliseconds). */
typedef struct bf_cuda_timing {
    double kernel_ms;   /* fit kernel(s) only: guess + LM + covariance */
    double total_ms;    /* whole call including copies */
    uint32_t launches;  /* fit kernel launches */
    int32_t group_lanes;
    int32_t grid;
    int32_t blocks_per_sm;
    double guess_ms;      /* data-only guess kernel(s) */
    double lm_ms;         /* LM kernel(s) */
    double covariance_ms; /* covariance kernel(s) */
    uint32_t batches;     /* device batches (chunks) the call ran */
} bf_cuda_timing;

const char *bf_cuda_last_error(void);
/* 1 when an sm_100-class device is present and usable. */
int bf_cuda_available(void);
int bf_cuda_version(void); /* library version, 100 * major + minor */

int bf_cuda_context_create(int device, bf_cuda_context **out);
void bf_cuda_context_destroy(bf_cuda_context *ctx);

/* Reference defaults for `model` under `policy`, bounds set to -inf/+inf. */
int bf_cuda_default_options(int32_t model, uint32_t policy, bf_solver_options *out);

/* Synchronous fit (submit + wait). */
int bf_cuda_fit(bf_cuda_context *ctx, const bf_fit_args *args, const bf_fit_outputs *out);

/* Asynchronous fit: the call returns once the work is queued on the GPU.  The
 * input and output buffers must stay valid and untouched until bf_cuda_wait. */
int bf_cuda_submit(bf_cuda_context *ctx, const bf_fit_args *args, const bf_fit_outputs *out,
                   bf_cuda_pending **pending);
/* 1 when the submission has completed, 0 when still running, <0 on error. */
int bf_cuda_ready(bf_cuda_pending *pending);
/* Waits, releases `pending` and returns the submission's result code. */
int bf_cuda_wait(bf_cuda_pending *pending);

/* Data-only guesses only (initial_guess<float,Model> per row); params[N*P] and
 * guess_status[N] (0 success, 1 invalid_input, 2 no_peak, 3 insufficient_peaks). */
int bf_cuda_guess(bf_cuda_context *ctx, int32_t model, uint64_t n, uint32_t m, const float *x,
                  const float *y, int32_t memory, float *params, int32_t *guess_status);

int bf_cuda_last_timing(bf_cuda_context *ctx, bf_cuda_timing *out);

/* Pinned host memory for BF_MEMORY_HOST calls that should overlap copies. */
int bf_cuda_host_alloc(size_t bytes, void **out);
int bf_cuda_host_free(void *ptr);

/* Largest M bf_cuda_fit takes for `model`.  With group_lanes 0, spectra of 6,144
 * points or more, and any that do not fit the group kernels' shared-memory layouts,
 * run one CTA (128 threads) per fit, reading x and y
 * through L2, with a long-spectrum guess; they take float32 y. */
uint32_t bf_cuda_max_points(int32_t model);

/* ---- Mixed batches --------------------------------------------------------
 * Many fit calls of different models and M run together: one persistent launch
 * per kernel (guess, LM, covariance) claims the fits of every segment from a
 * device work queue.  A segment is exactly one bf_cuda_fit call (one model, one
 * shared x[M], fit-major y[N*M], p0 or NULL, bounds, options, outputs), so each
 * segment is the reference's fit_batch<Model> / _core.fit call
 * (include/batchfit/metal/batch.hpp:268-310, python/bindings.cpp:200-207); the
 * reference has no call that mixes them.  Every pointer is device memory
 * (args.memory == BF_MEMORY_DEVICE); M may go up to bf_cuda_batch_max_points().
 * args.group_lanes 0 takes the tuned lanes per fit for (model, M)
 * (bf_cuda_autotune, else a built-in table); 8, 16 or 32 forces a width.
 * Results of a segment do not depend on the other segments in the batch. */
typedef struct bf_batch_segment {
    bf_fit_args args;
    bf_fit_outputs out;
} bf_batch_segment;

/* Flags of bf_cuda_fit_batch. */
#define BF_BATCH_FIXED_MAPPING 1u /* the plain mapping: one fit per warp (32 lanes), segments in call order */
#define BF_BATCH_NO_GRAPH 2u      /* launch the kernels one by one (per-kernel timing) instead of a graph replay */

/* Synchronous: returns when every segment's outputs are written.  Batches under
 * 32,768 fits replay a CUDA graph captured on the context (the LM kernels of the
 * batch's own (model, lanes) types enabled); larger ones launch their kernels
 * directly.  Either way the results are the same. */
int bf_cuda_fit_batch(bf_cuda_context *ctx, const bf_batch_segment *segments, uint32_t count, uint32_t flags);
uint32_t bf_cuda_batch_max_points(void);

/* Lanes per fit by (model, M bucket); bucket b holds M nearest 64 * 2^b
 * (b = 0..7: 64 ... 8192).  No counterpart in the reference, which maps one fit
 * per thread or per SIMD-group by a compile-time choice
 * (include/batchfit/metal/batch.hpp:268-310, KernelVariant). */
typedef struct bf_tuning {
    int32_t lanes[4][8];
    double lm_ms[4][8][3]; /* measured LM-kernel time per (model, bucket, 8/16/32 lanes); 0 if untimed */
    int32_t tuned;         /* 1 after bf_cuda_autotune or bf_cuda_set_tuning */
} bf_tuning;
/* Times the LM kernel for every (model, bucket) at 8, 16 and 32 lanes per fit on
 * seeded synthetic spectra generated on the device and keeps the fastest width.
 * Takes a few hundred milliseconds; later batches on the context use the result. */
int bf_cuda_autotune(bf_cuda_context *ctx, bf_tuning *out);
int bf_cuda_get_tuning(bf_cuda_context *ctx, bf_tuning *out);
int bf_cuda_set_tuning(bf_cuda_context *ctx, const bf_tuning *in);

/* ---- Serving: continuous batching of fit requests --------------------------
 * No counterpart in the reference, whose submit_batch queues one batch per context
 * and accepts no new work until it is collected (include/batchfit/metal/batch.hpp:
 * 198-217,253-264).  A server owns one GPU, a device-memory budget and a scheduler
 * thread.  Each request is one fit call in host memory (args->memory ==
 * BF_MEMORY_HOST; M up to bf_cuda_batch_max_points()).  Requests are admitted in
 * arrival order while their device buffers fit the budget, copied in, and
 * coalesced into mixed batches (bf_cuda_fit_batch's kernels).  Up to two batches
 * are on the GPU at once, on two streams: requests that arrive while a batch runs
 * form the next one, which starts as soon as they are copied in and overlaps the
 * running batch's tail.  A batch grows to about 1 ms of predicted device time; a
 * request predicted to take longer runs in a batch of its own, and smaller requests
 * that arrive after it may start before it.  At most one slot runs such a large
 * batch, launched with kernels sized for three quarters of the GPU's blocks, so
 * that short batches on the other slot always find room on every SM; a large
 * request alone runs on bf_cuda_fit's kernels (rows staged in shared memory) where
 * its M allows.  Outputs are
 * copied into the request's host buffers, which stay owned by the caller and must
 * stay valid until the request completes.  A
 * request's result is the one bf_cuda_fit_batch or bf_cuda_fit gives for it;
 * batch-mates only change its lanes per fit (so results agree within the parity
 * tolerances). */
typedef struct bf_server bf_server;

typedef struct bf_server_options {
    uint64_t memory_budget;  /* device bytes for admitted requests; 0 = 150 GB (capped by free memory) */
    uint64_t max_batch_fits; /* fits per launch; 0 = no limit */
    uint32_t batch_flags;    /* BF_BATCH_* of every launch */
    uint32_t max_in_flight;  /* batches on the GPU at once, 1 or 2; 0 = 2 */
} bf_server_options;

typedef struct bf_server_stats {
    uint64_t submitted, completed, failed, fits_completed, batches;
    uint64_t memory_in_use, memory_peak, memory_budget; /* bytes charged to admitted requests */
    uint64_t max_batch_requests;                        /* most requests in one launch */
    double gpu_ms;                                      /* summed device time of the mixed batches (not of
                                                           large requests run alone on the single-call kernels) */
} bf_server_stats;

int bf_server_create(int device, const bf_server_options *options, bf_server **out);
/* Stops taking requests, completes every submitted one, then frees the server. */
void bf_server_destroy(bf_server *server);
/* Queues a request; *ticket identifies it.  Fails (and queues nothing) when the
 * request is invalid or needs more device memory than the whole budget. */
int bf_server_submit(bf_server *server, const bf_fit_args *args, const bf_fit_outputs *out, uint64_t *ticket);
/* 1 when the request has completed, 0 while pending, -BF_ERR_INVALID_ARGUMENT for an unknown ticket. */
int bf_server_poll(bf_server *server, uint64_t ticket);
/* Waits for the request, releases its ticket and returns its result code;
 * *latency_ms (optional) = submit to outputs written. */
int bf_server_wait(bf_server *server, uint64_t ticket, double *latency_ms);
int bf_server_get_stats(bf_server *server, bf_server_stats *out);
/* Cancels a request that has not been admitted yet: returns 1 when it is cancelled
 * (its wait returns BF_ERR_CANCELLED), 0 when it is already admitted or finished
 * (it completes normally), -BF_ERR_INVALID_ARGUMENT for an unknown ticket. */
int bf_server_cancel(bf_server *server, uint64_t ticket);
/* Failure injection for tests of the failure handling, on the host: the next
 * `count` admissions fail as if the device allocation had run out of memory.  Such
 * a request completes with BF_ERR_CUDA, its bytes return to the budget and the
 * server carries on with the other requests (a real out-of-memory allocation is
 * handled the same way). */
int bf_server_fail_allocations(bf_server *server, uint32_t count);

/* ---- NPY streaming -----------------------------------------------------------
 * Out-of-core fits straight from .npy files: the reference's metal::fit_npy
 * (include/batchfit/metal/pipeline.hpp:49-67) behind its batchfit_fit_npy tool
 * (tools/fit_npy.cpp:20-121).  x_path holds x[M], y_path y[N,M] (fit-major, read
 * in chunks, never whole), initial_path (or NULL for data-only guesses) p0[N,P];
 * float32 or float64 (converted to float32), C order.  output_dir must not exist;
 * it receives parameters.npy (<f4 [N,P]), chi_squared.npy (<f4 [N]), status.npy
 * and iterations.npy (<u4 [N]) as the reference tool writes them, plus
 * covariance.npy, standard_errors.npy and uncertainty_status.npy with
 * uncertainties.  On failure the directory is removed. */
typedef struct bf_npy_options {
    int32_t model;           /* BF_MODEL_* */
    int32_t uncertainties;
    uint64_t chunk_fits;     /* fits per chunk; 0 = about 128 MB of y */
    uint32_t in_flight;      /* pinned chunks being read or fitted at once, 1..3; 0 = 3 */
    bf_solver_options solver;
} bf_npy_options;
typedef struct bf_npy_stats {
    uint64_t fits, chunks, chunk_fits;
    double wall_seconds, read_seconds, fit_seconds, write_seconds;
} bf_npy_stats;
int bf_cuda_fit_npy(bf_cuda_context *ctx, const char *x_path, const char *y_path, const char *initial_path,
                    const char *output_dir, const bf_npy_options *options, bf_npy_stats *stats);
/* Header of an .npy file: dtype 0 <f4, 1 <f8, 2 <u4; rank 1 or 2; shape[1] = 0 for
 * rank 1 (npy::inspect, src/cpu/npy.cpp:88-91).  Host only: needs no GPU. */
int bf_npy_inspect(const char *path, int32_t *dtype, int32_t *rank, uint64_t *shape);

/* ---- Physical units -----------------------------------------------------------
 * Fits of float64 data in normalised coordinates: the reference's struct
 * Coordinates (include/batchfit/coordinates.hpp:15-113).  Per call, x is centred on
 * the midpoint of its range and scaled by the half range; per fit, y is scaled by
 * its largest |y| (1 when all zero); both in double, then rounded to float32 for
 * the fit.  p0 (physical units, or NULL for data-only guesses on the normalised
 * data) is normalised the same way.  Bounds in `options` are in fitted
 * (normalised) units, as the reference requires.  Outputs come back in physical
 * units in double: parameters, chi-squared (x y_scale^2), covariance (T C T^T with
 * the reference's transform) and standard errors (square roots of its diagonal,
 * NaN without a covariance).  Non-finite inputs or a zero x range are refused
 * with BF_ERR_INVALID_ARGUMENT.  Device memory only. */
typedef struct bf_physical_args {
    int32_t model;
    uint64_t n;
    uint32_t m;
    const double *x;  /* [M] */
    const double *y;  /* [N*M] fit-major */
    const double *p0; /* [N*P] physical units, or NULL */
    int32_t uncertainties;
    int32_t group_lanes; /* 0 = tuned choice */
    bf_solver_options options;
} bf_physical_args;
typedef struct bf_physical_outputs {
    double *params;             /* [N*P] physical units */
    int32_t *status;            /* [N] */
    uint32_t *iterations;       /* [N] */
    double *chi2;               /* [N] physical units */
    double *covariance;         /* [N*P*P] when uncertainties */
    double *standard_errors;    /* [N*P] when uncertainties */
    int32_t *uncertainty_status;/* [N] when uncertainties */
} bf_physical_outputs;
int bf_cuda_fit_physical(bf_cuda_context *ctx, const bf_physical_args *args, const bf_physical_outputs *out);

/* A fit that needs no allocation of its own.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a host whose memory pool already owns
 * the whole device, a real-time pipeline that reserves every buffer up front and
 * forbids allocation while it runs, or a library callback that may only enqueue
 * work on a stream it was given.  Every pointer in `args` and `out` is device
 * memory of the current device (args->memory must be BF_MEMORY_DEVICE) and y is
 * float32 (args->y_format must be BF_Y_FLOAT32); anything else is rejected with
 * BF_ERR_INVALID_ARGUMENT.  The work is enqueued on `stream` (a cudaStream_t;
 * NULL = the default stream) and the call returns without waiting -- synchronise
 * the stream before reading the outputs.
 * The kernels' only scratch (the work counter and the data-only guesses) lives in
 * a 4 MiB static device array that every GPU loading this library holds until the
 * process exits.  With p0 == NULL, N is limited to the guesses that fit it --
 * 349,504 fits for P=3, 262,128 for P=4, 131,064 for P=8 -- and larger N is
 * rejected with BF_ERR_INVALID_ARGUMENT; with p0 given, N is not limited.
 * Every call looks up the array's device address in the calling thread's current
 * context (a host-side lookup that allocates nothing).  The first call in a context
 * loads the library's module and kernels, which places the array and the kernel
 * code in device memory: make that first call -- a call with N == 0 loads
 * everything for its model and M and launches nothing -- before a pool reserves
 * the whole device, or set CUDA_MODULE_LOADING=EAGER; and make it before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents (the work counter is cleared by every call): calls whose work overlaps
 * on the GPU race, so serialise them (one stream, or wait between calls).  No
 * context is needed. */
int bf_cuda_fit_noalloc(const bf_fit_args *args, const bf_fit_outputs *out, void *stream);

/* Roofline denominators measured on the context's device: dependent-chain
 * throughput of FP32 FMA (2 flops each), FP64 FMA, and the MUFU ex2 / rcp
 * approximations.  No reference counterpart (the reference has no roofline). */
typedef struct bf_cuda_peaks {
    double fp32_tflops;
    double fp64_tflops;
    double mufu_ex2_gops;
    double mufu_rcp_gops;
} bf_cuda_peaks;
int bf_cuda_measure_peaks(bf_cuda_context *ctx, bf_cuda_peaks *out);

#ifdef __cplusplus
}
#endif
#endif
