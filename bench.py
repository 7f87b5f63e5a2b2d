"""Benchmark: batched bounded-LM pseudo-Voigt fitting on B200.

Workload (one step): 1,000,000 pseudo-Voigt fits (amplitude, center, FWHM,
mixing) at M=512 on x = linspace(-10, 10, 512), float32, data-only guesses on the
GPU (p0=None), bounds [0,-10,1e-3,0]/[inf,10,10,1], uncertainties=True.  Seeded
synthetic spectra with the configuration's distributions (A~U[0.5,5], c~U[-6,6],
FWHM~logU[0.1,3], mixing~U[0,1], noise sigma = 1% of A).  y is 2.048 GB per GPU,
larger than L2 (126 MB), so no L2 flush is needed between steps.

* value     fits/s with x, y resident in HBM (one fit-kernel launch per step).
* e2e       the same fits through the C ABI from pinned host buffers: host->device
            copies, kernels and device->host result copies inside each step.
* accuracy  a 20,000-fit sample of the step's outputs against the float64 oracle.
* mixed, serving, configs  (N=1) the uneven mixed-model batch, the served stream,
            and the small-Lorentzian and two-Lorentzian-cube workloads with their
            accuracy against the float64 oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

N > 1 is launched under torch.distributed.run: every rank fits its own batch
(weak scaling, no data-path collective); time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fits/s at ≤1e-4 rel err vs FP64; p50/p99 latency, served vs plain on one B200"
MODEL, M, P = "pseudo_voigt", 512, 4
WORKLOAD = "pseudo_voigt_plain: 1M pseudo-Voigt fits, M=512, float32, p0=None, uncertainties=True"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) of the LM kernel per fit, from the committed ncu capture
# of the same kernel on 100,000 fits (profiles/fit_kernels_pv512_100k.md): 206.46 MB
# read + 4.45 MB written.  Traffic grows with the fits processed, so the bench scales
# it to the launch's fit count.
TRAFFIC_BYTES_PER_FIT = (206.462464e6 + 4.445696e6) / 100_000


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("cuda", "reference"), default="cuda")
    ap.add_argument("--fits", type=int, default=1_000_000, help="fits per GPU per step")
    ap.add_argument("--points", type=int, default=512,
                    help="points per spectrum (512 is the benchmark workload; a long M runs one CTA per fit)")
    ap.add_argument("--cpu-seconds", type=float, default=9.0, help="CPU-baseline sample budget per precision")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the uneven mixed-model batch section")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream section")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the small-Lorentzian and two-Lorentzian-cube section")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers --
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "cuda" else "gloo"
        if backend == "nccl":
            import torch

            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value, world, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sms, maxes, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxes.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(sms)}


HBM_FALLBACK_GBS = 6650.0  # an earlier copy-bandwidth measurement on a B200


def measured_peaks():
    try:
        with open(PEAKS_PATH) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def hbm_peak():
    """(GB/s, source): MEASURED_PEAKS.json's hbm_gbs, else the fallback."""
    mp = measured_peaks()
    if mp.get("hbm_gbs"):
        return float(mp["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return HBM_FALLBACK_GBS, "fallback 6650 GB/s (MEASURED_PEAKS.json absent; of fallback)"


# ------------------------------------------------------------- CPU legs --
def cpu_reference_rate(w, seconds_budget, dtype=np.float32):
    """The reference's own CPU path (oracle/_ref: guesses + cpu::fit_batch with
    uncertainties) on all host threads, over a bounded sample of the workload.
    Returns the rate with the data-only guesses included (what one fit call costs)
    and, for the compiled reference, the rate of fit_batch alone (guesses excluded,
    as the reference's own CPU timings are taken) and of the guesses alone."""
    from oracle import pyoracle

    if pyoracle.ref_available():
        kind, run = "reference", lambda n: pyoracle.fit("ref", MODEL, w.x, w.y[:n], None, w.lower, w.upper, dtype,
                                                        uncertainties=True)
        cores = int(pyoracle.load_ref().bfref_hardware_concurrency())
    else:
        kind, run = "port", lambda n: pyoracle.fit("port", MODEL, w.x, w.y[:n], None, w.lower, w.upper, dtype,
                                                   uncertainties=True)
        cores = 1
    n = min(2000, w.y.shape[0])
    t0 = time.perf_counter()
    run(n)  # warm-up and size probe
    per_fit = (time.perf_counter() - t0) / n
    n = int(min(w.y.shape[0], max(n, seconds_budget / 3 / max(per_fit, 1e-9))))
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        out = run(n)
        runs.append((time.perf_counter() - t0, out.guess_seconds, out.fit_seconds))
    sec, guess_s, fit_s = sorted(runs)[1]  # the median call
    res = {"value": n / sec, "unit": "fits/s", "cores": cores, "kind": kind,
           "sample": f"{n} fits of the same workload ({np.dtype(dtype).name} reference path incl. data-only guesses "
                     f"and covariance), median of 3 after a warm-up"}
    if kind == "reference" and fit_s > 0:
        res["fit_only_value"] = n / fit_s
        res["guess_only_value"] = n / guess_s if guess_s > 0 else None
    return res


def accuracy_sample(w, res_np, n=20000):
    from batchfit_b200 import accuracy
    from oracle import pyoracle

    n = min(n, w.y.shape[0])
    impl = "ref" if pyoracle.ref_available() else "port"
    ref = pyoracle.fit(impl, MODEL, w.x, w.y[:n], None, w.lower, w.upper, np.float64, uncertainties=True)
    counted = pyoracle.fit("port", MODEL, w.x, w.y[:2000], None, w.lower, w.upper, np.float64, count_passes=True)
    s = accuracy.summarize(MODEL, w.x, w.y[:n], res_np["params"][:n], res_np["status"][:n], res_np["chi2"][:n],
                           ref.params, ref.status, ref.chi2)
    us_agree = float((res_np["ustatus"][:n] == ref.uncertainty_status).mean())
    c = counted.counters
    passes = {"linearize": c.linearize_passes / 2000, "cost": c.cost_passes / 2000, "iterations": c.iterations / 2000}
    return {"oracle": f"float64 reference CPU path ({impl}) on the first {n} fits",
            "status_agreement": round(s["status_agreement"], 6),
            "within_tol_fraction": round(s["within_tol_fraction"], 6),
            "chi2_within_fraction": round(s["chi2_within_fraction"], 6),
            "param_err_max": s["param_err_max"], "param_err_p999": s["param_err_p999"],
            "chi2_err_max": s["chi2_err_max"], "uncertainty_status_agreement": round(us_agree, 6),
            "param_tol": 1e-4, "chi2_tol": 1e-5}, passes


# ------------------------------------------------------- mixed and serving --
def percentile(values, q):
    if not values:
        return None
    v = sorted(values)
    return v[min(len(v) - 1, max(0, math.ceil(q / 100.0 * len(v)) - 1))]


def mixed_section(ctx, dev):
    """65,536 fits of mixed models, per-fit M ~ logU[64,4096] on linspace(-10,10,M):
    one request per (model, M) sharing its x -- what the reference's one-x-per-call
    API takes.  Batched (one persistent launch per kernel, autotuned lanes, graph
    replay) against the plain path: one bf_cuda_fit per request with one fit per
    warp (32 lanes), in request order."""
    import ctypes as C

    import torch

    import batchfit_b200 as bf
    from batchfit_b200 import _capi, accuracy, workloads
    from oracle import pyoracle

    w = workloads.mixed_stream(n=65_536, seed=4)
    groups = {}
    for i in np.lexsort((w.counts, w.models)):
        groups.setdefault((int(w.models[i]), int(w.counts[i])), []).append(int(i))
    segs, keep, reqs = [], [], []
    for (mid, m), idx in groups.items():
        rows = np.stack([w.y[w.offsets[i]:w.offsets[i] + m] for i in idx])
        x = w.x[w.offsets[idx[0]]:w.offsets[idx[0]] + m].copy()
        model = workloads.MODEL_NAMES[mid]
        lo, hi = (np.array(v, np.float32) for v in workloads.MIXED_BOUNDS[model])
        a, o, res, k = bf._device_segment(torch.from_numpy(x).to(dev), torch.from_numpy(rows).to(dev), model,
                                          None, (lo, hi), False, "parity", 0, None)
        segs.append(_capi.BatchSegment(a, o))
        keep.append((res, k))
        reqs.append((model, x, rows, lo, hi, res))
    arr = (_capi.BatchSegment * len(segs))(*segs)
    lib = _capi.load()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.autotune()
    tune_s = time.perf_counter() - t0
    n_fits = int(w.models.size)

    def batched(flags, reps=5):
        walls, devs = [], []
        for _ in range(2):
            _capi.check(lib.bf_cuda_fit_batch(ctx.handle, arr, len(segs), flags), "bf_cuda_fit_batch")
        for _ in range(reps):
            t = time.perf_counter()
            _capi.check(lib.bf_cuda_fit_batch(ctx.handle, arr, len(segs), flags), "bf_cuda_fit_batch")
            walls.append(time.perf_counter() - t)
            devs.append(ctx.timing().kernel_ms)
        return statistics.median(walls) * 1e3, statistics.median(devs)

    tuned_wall, tuned_dev = batched(0)
    split = None
    _capi.check(lib.bf_cuda_fit_batch(ctx.handle, arr, len(segs), _capi.BF_BATCH_NO_GRAPH), "bf_cuda_fit_batch")
    t = ctx.timing()
    split = {"guess_ms": round(t.guess_ms, 3), "lm_ms": round(t.lm_ms, 3), "covariance_ms": round(t.covariance_ms, 3)}
    fixed_wall, fixed_dev = batched(_capi.BF_BATCH_FIXED_MAPPING)
    # Results of the tuned batch for the accuracy sample.
    _capi.check(lib.bf_cuda_fit_batch(ctx.handle, arr, len(segs), 0), "bf_cuda_fit_batch")
    torch.cuda.synchronize()
    sample = [(model, x, rows[:1], lo, hi, res.params[:1].cpu().numpy(), res.status[:1].cpu().numpy(),
               res.chi2[:1].cpu().numpy()) for (model, x, rows, lo, hi, res) in reqs[::10]]
    # Plain: one call per request, one fit per warp, device memory.
    plain_dev = 0.0
    t = time.perf_counter()
    for sgm in segs:
        a = sgm.args
        a.group_lanes = 32
        ctx.fit(a, sgm.out)
        plain_dev += ctx.timing().total_ms
        a.group_lanes = 0
    plain_wall = (time.perf_counter() - t) * 1e3
    # Accuracy of the batched fits on a sample (the first fit of every tenth request).
    definite = agree = within = within32 = equivalent = converged = 0
    per_model = {m: [0, 0] for m in workloads.MODEL_NAMES}
    for model, x, y1, lo, hi, gp, gs, gc in sample:
        ref = pyoracle.fit("port", model, x, y1, None, lo, hi, np.float64)
        if ref.status[0] == 1:
            continue
        r32 = pyoracle.fit("port", model, x, y1, None, lo, hi, np.float32)
        s = accuracy.summarize(model, x, y1, gp, gs, gc, ref.params, ref.status, ref.chi2, 1e-4, 1e-5, x64=True)
        s32 = accuracy.summarize(model, x, y1, r32.params, r32.status, r32.chi2, ref.params, ref.status, ref.chi2,
                                 1e-4, 1e-5)
        definite += 1
        agree += s["status_agreement"]
        within += s["within_tol_fraction"]
        within32 += s32["within_tol_fraction"]
        if ref.status[0] in (0, 5) and gs[0] == ref.status[0]:
            converged += 1
            equivalent += s["within_or_equivalent_fraction"]
            per_model[model][0] += s["within_tol_fraction"]
            per_model[model][1] += 1
    del keep
    return {
        "workload": "mixed_stream: 65,536 fits, 25% per model, M~logU[64,4096] on linspace(-10,10,M), p0=None; "
                    f"{len(segs)} requests (one per model and M, sharing x)",
        "batched": {"fits_per_s": n_fits / (tuned_dev * 1e-3), "device_ms": round(tuned_dev, 3),
                    "call_ms": round(tuned_wall, 3), "kernels_no_graph": split,
                    "what": "autotuned lanes; persistent guess and covariance launches, one LM launch per (model, lanes) class type over three streams; direct launches (graph replay below 32,768 fits)"},
        "fixed_mapping": {"fits_per_s": n_fits / (fixed_dev * 1e-3), "device_ms": round(fixed_dev, 3),
                          "call_ms": round(fixed_wall, 3), "what": "one launch, every fit on one warp, request order"},
        "plain_per_request": {"fits_per_s": n_fits / (plain_dev * 1e-3), "device_ms": round(plain_dev, 3),
                              "call_ms": round(plain_wall, 3),
                              "what": "one bf_cuda_fit per request, one fit per warp (32 lanes)"},
        "speedup_vs_plain": {"device": round(plain_dev / tuned_dev, 2), "call": round(plain_wall / tuned_wall, 2)},
        "autotune_s": round(tune_s, 3),
        "accuracy": {"sample_fits": len(sample), "definite": definite,
                     "status_agreement": round(agree / max(definite, 1), 5),
                     "within_tol_fraction": round(within / max(definite, 1), 5),
                     "reference_float32_within_tol_fraction": round(within32 / max(definite, 1), 5),
                     "within_or_float32_equivalent": round(equivalent / max(converged, 1), 5),
                     "within_tol_by_model": {m: round(v[0] / max(v[1], 1), 5) for m, v in per_model.items()},
                     "note": "fits the float64 oracle leaves at max_iterations are excluded (no definite status)"},
    }


def configs_section(ctx, dev, steps=5, warmup=3):
    """The other fixed-shape configurations, fitted on the GPU (device-resident,
    p0=None, uncertainties, parity policy) and checked against the float64 oracle:
    the reference's small CPU case (1,000 Lorentzians, M=129) and the two-Lorentzian
    cube (262,144 spectra, M=1024; 5% pure-noise and 2% constant rows).  The
    reference's own float32 path on the same sample is reported beside it."""
    import ctypes as C

    import torch

    import batchfit_b200 as bf
    from batchfit_b200 import _capi, accuracy, workloads
    from oracle import pyoracle

    impl = "ref" if pyoracle.ref_available() else "port"
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    out = {}
    for w, sample in ((workloads.lorentzian_small(), 1000), (workloads.two_lorentzian_cube(), 2000)):
        n, m = w.y.shape
        p = {"lorentzian": 3, "two_lorentzian": 8}[w.model]
        opts = bf.solver_options(w.model, w.lower, w.upper, "parity")
        x_d, y_d = torch.from_numpy(w.x).to(dev), torch.from_numpy(w.y).to(dev)
        o = {"params": torch.empty((n, p), dtype=torch.float32, device=dev),
             "status": torch.empty(n, dtype=torch.int32, device=dev),
             "iters": torch.empty(n, dtype=torch.int32, device=dev),
             "chi2": torch.empty(n, dtype=torch.float32, device=dev),
             "cov": torch.empty((n, p, p), dtype=torch.float32, device=dev),
             "se": torch.empty((n, p), dtype=torch.float32, device=dev),
             "ustatus": torch.empty(n, dtype=torch.int32, device=dev)}
        fa = _capi.FitArgs(workloads.MODEL_NAMES.index(w.model), n, m, dp(x_d), dp(y_d), None,
                           _capi.BF_MEMORY_DEVICE, 1, 0, opts)
        fo = _capi.FitOutputs(dp(o["params"]), dp(o["status"]), dp(o["iters"]), dp(o["chi2"]), dp(o["cov"]),
                              dp(o["se"]), dp(o["ustatus"]))
        for _ in range(warmup):
            ctx.fit(fa, fo)
        ms, split = [], {"guess_ms": [], "lm_ms": [], "covariance_ms": []}
        for _ in range(steps):
            ctx.fit(fa, fo)
            t = ctx.timing()
            ms.append(t.total_ms)
            for k in split:
                split[k].append(getattr(t, k))
        res = {k: v.cpu().numpy() for k, v in o.items()}
        k = min(sample, n)
        ref = pyoracle.fit(impl, w.model, w.x, w.y[:k], None, w.lower, w.upper, np.float64, uncertainties=True)
        r32 = pyoracle.fit(impl, w.model, w.x, w.y[:k], None, w.lower, w.upper, np.float32)
        # The float64 oracle run to much tighter tolerances: how far its own answer
        # moves (the part of the 1e-4 bar no solver can be held to).
        tight = pyoracle.fit(impl, w.model, w.x, w.y[:k], None, w.lower, w.upper, np.float64,
                             options=pyoracle.make_options(max_iterations=2000, gradient_tolerance=1e-16,
                                                           step_tolerance=1e-16, cost_tolerance=1e-18))
        s = accuracy.summarize(w.model, w.x, w.y[:k], res["params"][:k], res["status"][:k], res["chi2"][:k],
                               ref.params, ref.status, ref.chi2, x64=True, bounds=(w.lower, w.upper))
        s32 = accuracy.summarize(w.model, w.x, w.y[:k], r32.params, r32.status, r32.chi2, ref.params, ref.status,
                                 ref.chi2, x64=True, bounds=(w.lower, w.upper))
        s64 = accuracy.summarize(w.model, w.x, w.y[:k], tight.params, tight.status, tight.chi2, ref.params,
                                 ref.status, ref.chi2)
        codes, counts = np.unique(res["status"], return_counts=True)
        step_ms = statistics.median(ms)
        out[w.name] = {
            "fits": n, "points": m, "model": w.model, "fits_per_s": n / (step_ms * 1e-3),
            "ms_per_step": round(step_ms, 3),
            "kernels_ms": {k: round(statistics.median(v), 3) for k, v in split.items()},
            "status_counts": {str(int(c)): int(v) for c, v in zip(codes, counts)},
            "accuracy": {"oracle": f"float64 reference CPU path ({impl}) on the first {k} fits",
                         "status_agreement": round(s["status_agreement"], 6),
                         "within_tol_fraction": round(s["within_tol_fraction"], 6),
                         "params_within_fraction": round(s["params_within_fraction"], 6),
                         "chi2_within_fraction": round(s["chi2_within_fraction"], 6),
                         "param_err_max": s["param_err_max"], "param_err_p999": s["param_err_p999"],
                         "chi2_err_max": s["chi2_err_max"],
                         "uncertainty_status_agreement": round(
                             float((res["ustatus"][:k] == ref.uncertainty_status).mean()), 6),
                         "status_agreement_definite": round(s["status_agreement_definite"], 6),
                         "within_or_float32_equivalent": round(s["within_or_equivalent_fraction"], 6),
                         "reference_float32_within_tol_fraction": round(s32["within_tol_fraction"], 6),
                         "reference_float32_status_agreement": round(s32["status_agreement"], 6),
                         "reference_float32_status_agreement_definite": round(s32["status_agreement_definite"], 6),
                         "reference_float32_within_or_float32_equivalent":
                             round(s32["within_or_equivalent_fraction"], 6),
                         "float64_tight_vs_default_within_tol": round(s64["within_tol_fraction"], 6),
                         "float32_bounds": {
                             "what": "over the oracle-converged fits, relative to the parameter errors' "
                                     "denominators: first_order = (J^T J)^-1 J^T of u32 (|y|+|f|), how far float32 "
                                     "evaluation moves the fixed point J^T r = 0; chi2_resolution = "
                                     "sqrt(eps (J^T J)^-1_kk), how far parameters move while chi2 stays within its "
                                     "float32 evaluation error eps",
                             "first_order_median": s["first_order_median"],
                             "first_order_below_tol_fraction": round(s["first_order_below_tol_fraction"], 6),
                             "within_tol_where_first_order_below_tol": s["within_tol_where_first_order_below_tol"],
                             "reference_float32_within_tol_where_first_order_below_tol":
                                 s32["within_tol_where_first_order_below_tol"],
                             "chi2_resolution_median": s["chi2_resolution_median"],
                             "chi2_resolution_below_tol_fraction": round(s["chi2_resolution_below_tol_fraction"], 6)},
                         "param_tol": 1e-4, "chi2_tol": 1e-5},
        }
        del x_d, y_d, o
        torch.cuda.empty_cache()
    return out


def serving_section(lib):
    """Poisson arrivals of fit requests (N ~ logU[1,50000], M ~ logU[64,2048], random
    model, half with uncertainties, p0=None) at several rates: the continuous-
    batching server against plain per-request calls in arrival order (one fit per
    warp).  Latency = arrival to outputs in host memory."""
    import ctypes as C

    import batchfit_b200 as bf
    from batchfit_b200 import _capi, workloads

    pinned = []

    def alloc(shape):
        nbytes = int(np.prod(shape)) * 4
        ptr = C.c_void_p()
        _capi.check(lib.bf_cuda_host_alloc(nbytes, C.byref(ptr)), "bf_cuda_host_alloc")
        pinned.append(ptr)
        buf = (C.c_float * int(np.prod(shape))).from_address(ptr.value)
        return np.frombuffer(buf, np.float32).reshape(shape)

    t0 = time.perf_counter()
    pool = workloads.serving_pool(alloc=alloc)
    pool_s = time.perf_counter() - t0
    ctx = bf.context(0)

    def plain_call(r, x, y, bounds):
        p = 8 if r.model == "two_lorentzian" else 4 if r.model == "pseudo_voigt" else 3
        o = {k: np.empty(s, dt) for k, s, dt in (("params", (r.n, p), np.float32), ("status", r.n, np.int32),
                                                 ("iters", r.n, np.uint32), ("chi2", r.n, np.float32))}
        if r.uncertainties:
            o.update({"cov": np.empty((r.n, p, p), np.float32), "se": np.empty((r.n, p), np.float32),
                      "us": np.empty(r.n, np.int32)})
        opts = bf.solver_options(r.model, bounds[0], bounds[1], "parity")
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        args = _capi.FitArgs(bf.MODELS[r.model], r.n, x.size, ptr(x), ptr(y), None, _capi.BF_MEMORY_HOST,
                             int(r.uncertainties), 32, opts)
        outs = _capi.FitOutputs(ptr(o["params"]), ptr(o["status"]), ptr(o["iters"]), ptr(o["chi2"]),
                                ptr(o.get("cov")), ptr(o.get("se")), ptr(o.get("us")))
        ctx.fit(args, outs)

    # Both arms warm up on the largest requests first (staging buffers, graphs).
    warm = [workloads.ServingRequest(0.0, model, workloads.SERVING_M[-1], pool.n_max, True)
            for model in workloads.MODEL_NAMES]
    for r in warm:
        x = pool.x[(r.model, r.m)]
        lo, hi = (np.array(v, np.float32) for v in workloads.MIXED_BOUNDS[r.model])
        plain_call(r, x, pool.y[(r.model, r.m)][:r.n], (lo, hi))
    out = []
    for k, (rate, duration) in enumerate(((10, 4.0), (100, 3.0), (1000, 2.0), (2000, 2.0))):
        stream = workloads.serving_stream(rate, duration, seed=50 + k)
        fits = sum(r.n for r in stream)

        def views(r):
            x = pool.x[(r.model, r.m)]
            y = pool.y[(r.model, r.m)][:r.n]
            lo, hi = (np.array(v, np.float32) for v in workloads.MIXED_BOUNDS[r.model])
            return x, y, (lo, hi)

        # Served.
        with bf.Server() as server:
            for r in warm:
                x, y, bounds = views(r)
                server.submit(x, y, r.model, None, bounds, uncertainties=True).result()
            base = server.stats()
            tickets = []
            start = time.perf_counter()
            for r in stream:
                delay = start + r.arrival - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                x, y, bounds = views(r)
                tickets.append(server.submit(x, y, r.model, None, bounds, uncertainties=r.uncertainties))
            for tk in tickets:
                tk.result()
            end = time.perf_counter()
            st = server.stats()
        lat = [tk.latency_ms for tk in tickets]
        served = {"p50_ms": round(percentile(lat, 50), 3), "p99_ms": round(percentile(lat, 99), 3),
                  "fits_per_s": fits / (end - start), "batches": st["batches"] - base["batches"],
                  "max_requests_per_batch": st["max_batch_requests"],
                  "gpu_busy_ms": round(st["gpu_ms"] - base["gpu_ms"], 2),
                  "memory_peak_gb": round(st["memory_peak"] / 1e9, 3)}
        # Plain: requests served one at a time in arrival order; stops taking new
        # requests after 6x the stream's duration (the rest are reported unserved).
        lat_p, served_fits, unserved = [], 0, 0
        start = time.perf_counter()
        for r in stream:
            now = time.perf_counter() - start
            if now > 6 * duration + 2.0:
                unserved += 1
                continue
            if r.arrival > now:
                time.sleep(r.arrival - now)
            x, y, bounds = views(r)
            plain_call(r, x, y, bounds)
            done = time.perf_counter() - start
            lat_p.append((done - r.arrival) * 1e3)
            served_fits += r.n
        end_p = time.perf_counter() - start
        plain = {"p50_ms": round(percentile(lat_p, 50), 3) if lat_p else None,
                 "p99_ms": round(percentile(lat_p, 99), 3) if lat_p else None,
                 "fits_per_s": served_fits / end_p, "unserved_requests": unserved}
        out.append({"rate_per_s": rate, "duration_s": duration, "requests": len(stream), "fits": fits,
                    "served": served, "plain": plain,
                    "p99_ratio_plain_over_served": round(plain["p99_ms"] / served["p99_ms"], 2)
                    if plain["p99_ms"] else None,
                    "throughput_ratio_served_over_plain": round(served["fits_per_s"] / plain["fits_per_s"], 2)})
    for ptr in pinned:
        lib.bf_cuda_host_free(ptr)
    return {"stream": "Poisson arrivals; N~logU[1,50000], M~logU[64,2048] (8 log-spaced values), random model, "
                      "half with uncertainties, p0=None; inputs in pinned host memory",
            "pool_setup_s": round(pool_s, 2), "rates": out,
            "plain_what": "bf_cuda_fit per request in arrival order (host buffers, one fit per warp)",
            "served_what": "bf_server: HBM-budget admission, coalesced mixed batches, two batches in flight"}


def summary_of(line):
    """The line's key figures, repeated compactly as its last key: a reader that
    keeps only the end of a long line still sees them."""
    def pick(d, *path):
        for k in path:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    out = {"fits_per_s": round(line["value"]), "e2e_fits_per_s": round(line["e2e"]["value"]),
           "ms_per_step": round(line["ms_per_step"], 3),
           "within_1e-4": pick(line, "accuracy", "within_tol_fraction"),
           "status_agreement": pick(line, "accuracy", "status_agreement"),
           "lm_fp32_frac": pick(line, "roofline", "frac"), "step_frac": pick(line, "roofline", "step_frac"),
           "cpu_f32_fits_per_s": pick(line, "cpu_baseline", "value"),
           "cpu_f64_fits_per_s": pick(line, "cpu_baseline", "value_f64")}
    cube = pick(line, "configs", "two_lorentzian_cube")
    if cube:
        out["cube"] = {"fits_per_s": round(cube["fits_per_s"]),
                       "status_definite": cube["accuracy"]["status_agreement_definite"],
                       "within_1e-4": cube["accuracy"]["within_tol_fraction"],
                       "within_or_f32_equivalent": cube["accuracy"]["within_or_float32_equivalent"],
                       "within_where_first_order_bound_small":
                           cube["accuracy"]["float32_bounds"]["within_tol_where_first_order_below_tol"]}
    mixed = line.get("mixed")
    if mixed:
        out["mixed"] = {"batched_ms": mixed["batched"]["device_ms"], "fixed_ms": mixed["fixed_mapping"]["device_ms"],
                        "status": mixed["accuracy"]["status_agreement"],
                        "within_or_f32_equivalent": mixed["accuracy"]["within_or_float32_equivalent"]}
    serving = line.get("serving")
    if serving:
        out["serving_p99_ms"] = {str(r["rate_per_s"]): [r["served"]["p99_ms"], r["plain"]["p99_ms"]]
                                 for r in serving["rates"]}
    return out


# -------------------------------------------------------------- arms --
def run_reference_arm(args, world, rank):
    from batchfit_b200 import workloads

    if rank != 0:
        return 0
    n = min(200_000, args.fits)
    w = workloads.pseudo_voigt_plain(n=n, m=M)
    from oracle import pyoracle

    impl = "ref" if pyoracle.ref_available() else "port"
    cores = int(pyoracle.load_ref().bfref_hardware_concurrency()) if impl == "ref" else 1
    # Size each step to a bounded sample of the workload (~1-2 s of CPU work).
    probe = min(2000, n)
    t0 = time.perf_counter()
    pyoracle.fit(impl, MODEL, w.x, w.y[:probe], None, w.lower, w.upper, np.float32, uncertainties=True)
    per_fit = (time.perf_counter() - t0) / probe
    sample = int(min(n, max(min(probe, n), 1.5 / max(per_fit, 1e-9))))
    for _ in range(args.warmup):
        pyoracle.fit(impl, MODEL, w.x, w.y[:sample], None, w.lower, w.upper, np.float32, uncertainties=True)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pyoracle.fit(impl, MODEL, w.x, w.y[:sample], None, w.lower, w.upper, np.float32, uncertainties=True)
        times.append(time.perf_counter() - t0)
    value = sample * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "fits_per_step": sample, "points": M, "model": MODEL,
                   "sample": "bounded sample of the same workload per step"},
        "cpu_baseline": {"value": value, "unit": "fits/s", "cores": cores,
                         "kind": "reference" if impl == "ref" else "port",
                         "sample": f"{sample} fits per step: the reference's float32 cpu::fit_batch with data-only "
                                   f"guesses and uncertainties on {cores} host threads"},
        "e2e": {"value": value, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_cuda_arm(args, world, rank, local):
    import ctypes as C

    import torch

    import batchfit_b200 as bf
    from batchfit_b200 import _capi, roofline, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workloads.pseudo_voigt_plain(n=args.fits, m=M, seed=2 + rank)
    n = w.y.shape[0]
    ctx = bf.context(local)
    opts = bf.solver_options(MODEL, w.lower, w.upper, "parity")
    x_d = torch.from_numpy(w.x).to(dev)
    y_d = torch.from_numpy(w.y).to(dev)
    out_d = {"params": torch.empty((n, P), dtype=torch.float32, device=dev),
             "status": torch.empty(n, dtype=torch.int32, device=dev),
             "iters": torch.empty(n, dtype=torch.int32, device=dev),
             "chi2": torch.empty(n, dtype=torch.float32, device=dev),
             "cov": torch.empty((n, P, P), dtype=torch.float32, device=dev),
             "se": torch.empty((n, P), dtype=torch.float32, device=dev),
             "ustatus": torch.empty(n, dtype=torch.int32, device=dev)}
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    d_args = _capi.FitArgs(2, n, M, dp(x_d), dp(y_d), None, _capi.BF_MEMORY_DEVICE, 1, 0, opts)
    d_outs = _capi.FitOutputs(dp(out_d["params"]), dp(out_d["status"]), dp(out_d["iters"]), dp(out_d["chi2"]),
                              dp(out_d["cov"]), dp(out_d["se"]), dp(out_d["ustatus"]))
    torch.cuda.synchronize()

    # ---- value: device-resident inputs ----
    for _ in range(args.warmup):
        ctx.fit(d_args, d_outs)
    barrier(world)
    torch.cuda.synchronize()
    step_ms, kernel_ms, launches = [], [], 0
    split = {"guess_ms": [], "lm_ms": [], "covariance_ms": []}
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            ctx.fit(d_args, d_outs)
            t = ctx.timing()
            step_ms.append(t.total_ms)
            kernel_ms.append(t.kernel_ms)
            for k in split:
                split[k].append(getattr(t, k))
            launches += t.launches
            lanes, grid, bps = t.group_lanes, t.grid, t.blocks_per_sm
    torch.cuda.synchronize()
    barrier(world)
    total_ms = max_over_ranks(sum(step_ms), world, dev)
    value = world * n * args.steps / (total_ms * 1e-3)

    # ---- e2e: pinned host buffers through the C ABI ----
    lib = _capi.load()
    host = {}

    def pinned(nbytes):
        ptr = C.c_void_p()
        _capi.check(lib.bf_cuda_host_alloc(nbytes, C.byref(ptr)), "bf_cuda_host_alloc")
        host[ptr.value] = nbytes
        return ptr

    hx, hy = pinned(w.x.nbytes), pinned(w.y.nbytes)
    C.memmove(hx, w.x.ctypes.data, w.x.nbytes)
    C.memmove(hy, w.y.ctypes.data, w.y.nbytes)
    o_bytes = {"params": n * P * 4, "status": n * 4, "iters": n * 4, "chi2": n * 4, "cov": n * P * P * 4,
               "se": n * P * 4, "ustatus": n * 4}
    ho = {k: pinned(v) for k, v in o_bytes.items()}
    h_args = _capi.FitArgs(2, n, M, hx, hy, None, _capi.BF_MEMORY_HOST, 1, 0, opts)
    h_outs = _capi.FitOutputs(ho["params"], ho["status"], ho["iters"], ho["chi2"], ho["cov"], ho["se"],
                              ho["ustatus"])
    for _ in range(max(1, args.warmup)):
        ctx.fit(h_args, h_outs)
    barrier(world)
    e2e_ms = []
    for _ in range(args.steps):
        ctx.fit(h_args, h_outs)
        e2e_ms.append(ctx.timing().total_ms)
    barrier(world)
    e2e_total = max_over_ranks(sum(e2e_ms), world, dev)
    e2e_value = world * n * args.steps / (e2e_total * 1e-3)
    h2d = w.x.nbytes + w.y.nbytes
    d2h = sum(o_bytes.values())

    # Opt-in half-precision y (BF_Y_FLOAT16): the same step with y rounded to binary16
    # by the caller, half the host-to-device bytes.  Not the headline (it fits
    # different, rounded values); reported beside it.
    y16 = w.y.astype(np.float16)  # kept alive until the copy into pinned memory is done
    hy16 = pinned(y16.nbytes)
    C.memmove(hy16, y16.ctypes.data, y16.nbytes)
    del y16
    h16_args = _capi.FitArgs(2, n, M, hx, hy16, None, _capi.BF_MEMORY_HOST, 1, 0, opts, _capi.BF_Y_FLOAT16)
    try:
        ctx.fit(h16_args, h_outs)
    except ValueError as e:  # long spectra (one CTA per fit) take float32 y only
        e2e16 = {"unavailable": str(e)}
    else:
        for _ in range(max(1, args.warmup)):
            ctx.fit(h16_args, h_outs)
        barrier(world)
        e2e16_ms = []
        for _ in range(args.steps):
            ctx.fit(h16_args, h_outs)
            e2e16_ms.append(ctx.timing().total_ms)
        barrier(world)
        e2e16_total = max_over_ranks(sum(e2e16_ms), world, dev)
        e2e16 = {"value": world * n * args.steps / (e2e16_total * 1e-3), "unit": "fits/s",
                 "h2d_bytes_per_step": w.x.nbytes + w.y.size * 2, "d2h_bytes_per_step": d2h,
                 "what": "opt-in BF_Y_FLOAT16: y given as binary16 (rounded by the caller), converted exactly to "
                         "float32 on the GPU; half the host-to-device bytes"}
    # The float32 step's outputs are read below: run it once more after the fp16 runs.
    ctx.fit(h_args, h_outs)

    # Host and device paths must agree bit for bit.
    res_np = {k: np.ctypeslib.as_array(C.cast(ho[k], C.POINTER(C.c_uint8)), (o_bytes[k],)).copy()
              for k in o_bytes}
    res_np = {"params": res_np["params"].view(np.float32).reshape(n, P),
              "status": res_np["status"].view(np.int32), "chi2": res_np["chi2"].view(np.float32),
              "ustatus": res_np["ustatus"].view(np.int32)}
    same = bool(np.array_equal(res_np["params"], out_d["params"].cpu().numpy(), equal_nan=True))
    for ptr in list(host):
        lib.bf_cuda_host_free(C.c_void_p(ptr))

    if rank != 0:
        return 0
    # ---- accuracy, roofline, CPU baseline (rank 0) ----
    acc, passes = accuracy_sample(w, res_np)
    peaks = ctx.measure_peaks()
    flops, mufu = roofline.fit_work(MODEL, M, passes["linearize"], passes["cost"], True)
    # The LM kernel is the dominant launch: every model evaluation of the fit runs in
    # it, so its algorithmic work is divided by its own event-timed duration.
    k_ms = statistics.mean(split["lm_ms"])
    all_ms = statistics.mean(kernel_ms)
    g_ms = statistics.mean(split["guess_ms"])
    achieved_tf = flops * n / (k_ms * 1e-3) / 1e12
    mufu_rate = mufu * n / (k_ms * 1e-3) / 1e9
    mufu_peak = min(peaks.mufu_ex2_gops, peaks.mufu_rcp_gops)
    ideal_ms = max(flops * n / (peaks.fp32_tflops * 1e12), mufu * n / (mufu_peak * 1e9),
                   roofline.observation_bytes(M, P, True) * n / (hbm_peak()[0] * 1e9)) * 1e3
    hbm_gbs = roofline.observation_bytes(M, P, True) * n / (all_ms * 1e-3) / 1e9
    guess_gbs = 4 * M * n / (g_ms * 1e-3) / 1e9
    hbm_gbs_peak, hbm_source = hbm_peak()
    roof = {
        "bound": "fp32", "kernel": (f"lm_kernel<pseudo_voigt, {lanes} lanes>" if lanes != 128
                                    else "lm_cta_kernel<pseudo_voigt> (one CTA per fit)"),
        "achieved": round(achieved_tf, 3),
        "peak": round(peaks.fp32_tflops, 3), "unit": "TFLOP/s", "frac": round(achieved_tf / peaks.fp32_tflops, 4),
        "traffic": None if TRAFFIC_BYTES_PER_FIT is None else int(TRAFFIC_BYTES_PER_FIT * n),
        "peak_source": "measured in this run: FFMA microbenchmark on this GPU (bf_cuda_measure_peaks)",
        "ideal_ms": round(ideal_ms, 4), "lm_kernel_ms": round(k_ms, 4), "all_kernels_ms": round(all_ms, 4),
        "roofline_frac": round(ideal_ms / k_ms, 4),
        "step_frac": round(ideal_ms / all_ms, 4),
        "step_what": "ideal time (slowest of FP32, MUFU, HBM at measured peaks) / all kernels of the step",
        "kernels_ms": {"guess": round(g_ms, 4), "lm": round(k_ms, 4),
                       "covariance": round(statistics.mean(split["covariance_ms"]), 4)},
        "guess_hbm": {"achieved": round(guess_gbs, 1), "unit": "GB/s",
                      "frac": round(guess_gbs / hbm_gbs_peak, 4), "peak_source": hbm_source,
                      "what": "y bytes read by the guess kernel / its duration"},
        "mufu": {"achieved_gops": round(mufu_rate, 1), "peak_gops": round(mufu_peak, 1),
                 "frac": round(mufu_rate / mufu_peak, 4)},
        "hbm": {"achieved": round(hbm_gbs, 1), "peak": hbm_gbs_peak, "unit": "GB/s",
                "frac": round(hbm_gbs / hbm_gbs_peak, 4), "peak_source": hbm_source,
                "what": "observation bytes of the whole fit / all kernels' duration"},
        "work": {"flops_per_fit": round(flops), "mufu_per_fit": round(mufu), "oracle_passes": passes},
    }
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_reference_rate(w, args.cpu_seconds)
        # The float64 reference beside it (same inputs promoted), and the rates with
        # the data-only guesses excluded, as the reference's CPU timings are taken.
        c64 = cpu_reference_rate(w, args.cpu_seconds, np.float64)
        cpu["value_f64"] = c64["value"]
        cpu["sample_f64"] = c64["sample"]
        for key in ("fit_only_value", "guess_only_value"):
            if key in cpu:
                cpu[key + "_f32"] = cpu.pop(key)
            if key in c64:
                cpu[key + "_f64"] = c64[key]
    del y_d, out_d
    torch.cuda.empty_cache()
    # The mixed-batch and serving sections run at N=1 only (one GPU's batching and
    # serving; the scaling runs repeat the plain workload per GPU).
    mixed = None if args.no_mixed or world > 1 else mixed_section(ctx, dev)
    serving = None if args.no_serving or world > 1 else serving_section(lib)
    configs = None if args.no_configs or world > 1 else configs_section(ctx, dev)
    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "fits_per_gpu": n, "points": M, "model": MODEL, "uncertainties": True,
                   "p0": "None (GPU data-only guesses)", "policy": "parity", "group_lanes": lanes, "grid": grid,
                   "blocks_per_sm": bps, "l2": "inputs (2.048 GB/GPU) exceed L2; no flush",
                   "parallelism": f"replicas x{world} (independent fits, no collective)"},
        "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, math.ceil(0.99 * len(lat)) - 1)],
                       "what": "per-step (1M-fit batch) device time"},
        "e2e": {"value": e2e_value, "unit": "fits/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "host_device_match": same},
        "e2e_fp16_y": e2e16,
        "gpu_launches": launches,
        "accuracy": acc,
        "roofline": roof,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
        "mixed": mixed,
        "serving": serving,
        "configs": configs,
        "peaks_measured": {"fp32_tflops": round(peaks.fp32_tflops, 2), "fp64_tflops": round(peaks.fp64_tflops, 2),
                           "mufu_ex2_gops": round(peaks.mufu_ex2_gops, 1),
                           "mufu_rcp_gops": round(peaks.mufu_rcp_gops, 1)},
    }
    line["summary"] = summary_of(line)
    print(json.dumps(line), flush=True)
    return 0


def main():
    global M, WORKLOAD
    args = parse()
    if args.points != M:
        M = args.points
        WORKLOAD = WORKLOAD.replace("M=512", f"M={M}")
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            return run_reference_arm(args, world, rank)
        return run_cuda_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
