// Device work queue of a mixed batch: spectra of uneven M and mixed models fitted
// by one persistent launch per kernel (guess, LM, covariance).
//
// A batch is a list of segments.  A segment is n fits that share a model, M, an x
// grid, options and output arrays -- one call of the reference's fit API
// (python/bindings.cpp:200-207 takes one shared x per call).  The host planner
// splits every segment into runs and files each run under a work class: (model,
// lanes per fit, octave of M) for the LM kernel, (model, lanes, guess register
// width, octave of M) for the guess kernel.  Classes are ordered by cost per fit, largest first, and runs
// within a class by M, largest first, so the cheapest fits fill the tail.  A
// preparation kernel writes one work item per fit; the persistent kernels claim
// the items of a class through the class's atomic counter.
#pragma once

#include "bf_args.h"

namespace bf {

// Largest M of a batch segment: the guess kernel's per-warp sorting buffer holds
// two edge runs of up to 1024 samples (M/10 per side).
constexpr int kBatchMaxPoints = 10240;
constexpr int kBatchMaxSortWidth = 1024;
constexpr int kMaxClasses = 256; // >= 4 models x 3 widths x 14 octaves of M

struct Segment {
    FitArgs a;        // x, y, p0, outputs, n, m and options (a.p0 == guesses without user p0)
    XConst xc;        // filled on the device by the preparation kernel
    float *guesses;   // [n*P] data-only guesses, or nullptr when the caller gave p0
    int model;
    int pad;
};

// A class of work items that one code path (template instantiation) processes.
struct WorkClass {
    int model;
    int lanes;        // 8, 16 or 32 lanes per fit
    int v;            // guess classes: register sort width per lane (0 = shared-memory sort)
    int pad;
    long long begin;  // first work item of the class
    long long fits;   // work items in the class
};

// Fits [first, first+count) of one segment; items [start, start+count) of the queue.
struct WorkRun {
    int segment;
    int pad;
    long long first;
    long long count;
    long long start;
};

struct WorkItem {
    int segment;
    int fit; // index within the segment
};

// Counts of the batch in flight, read by the kernels from device memory so that a
// captured graph replays for every batch that fits the arena.
struct BatchHeader {
    int segments;
    int lm_classes;
    int guess_classes;
    int lm_runs;
    int guess_runs;
    int uncertain_segments; // segments with uncertainties (0: the covariance kernel exits)
    long long lm_items;
    long long guess_items;
};

// Kernel parameter block: device pointers into the batch arena.
struct BatchArgs {
    const BatchHeader *hdr;
    Segment *segs;
    const WorkClass *lm_classes, *guess_classes;
    const WorkRun *lm_runs, *guess_runs;
    WorkItem *lm_items, *guess_items;
    unsigned long long *counters; // [kMaxClasses] LM classes, then [kMaxClasses] guess classes
};

// LM work-class types: one kernel each, index model * 3 + (8 -> 0, 16 -> 1, 32 -> 2).
constexpr int kLmClassTypes = 12;
constexpr uint32_t kAllLmTypes = (1u << kLmClassTypes) - 1u;
inline int lm_class_type(int model, int lanes) { return model * 3 + (lanes == 8 ? 0 : lanes == 16 ? 1 : 2); }

// Side streams for the LM kernels of a batch: the kernels of different work-class
// types run on kLmStreams streams (the batch's own and these), so that one
// kernel's tail fills with the next kernel's blocks.
constexpr int kLmStreams = 3;
struct LmFork {
    cudaStream_t side[kLmStreams - 1] = {};
    cudaEvent_t fork = nullptr, join[kLmStreams - 1] = {};
};
cudaError_t create_lm_fork(LmFork &f);
void release_lm_fork(LmFork &f);

// Host entry points (bf_batch_kernels.cu).  Every launch goes to `stream` (and
// the fork's side streams) with a grid fixed by the device, so a captured sequence
// replays for any batch.  The LM kernels of the types in `lm_types` (bit per type)
// are launched; a captured pipeline holds all of them.
cudaError_t launch_batch_pipeline(const BatchArgs &b, int sms, cudaStream_t stream, cudaEvent_t guessed,
                                  cudaEvent_t fitted, const LmFork *fork, uint32_t lm_types = kAllLmTypes);
// The LM kernel of a work-class type (to find its node in a captured graph).
const void *batch_lm_function(int type);
// Guess code path (lanes, register width) for M; false when M/10 exceeds the
// sorting buffer.
bool batch_guess_shape(int m, int *lanes, int *v);
// Seeded synthetic spectra of `model` on x = linspace(-10, 10, m): the mixed
// workload's parameter distributions (amplitude U[0.5,5], center U[-6,6], FWHM
// log-uniform [0.1,3], mixing U[0,1]; a second Lorentzian for two_lorentzian) plus
// Gaussian noise of 1% of the amplitude.  Used by the autotuner.
cudaError_t launch_synthetic(int model, int m, long long n, unsigned seed, float *x, float *y,
                             cudaStream_t stream);

} // namespace bf
