"""Mixed batches: many fit calls of different models and M in one persistent launch.

* A segment's result in a mixed batch equals, bit for bit, the result of the same
  call alone through ``fit`` at the same lanes per fit (the kernels read x and y
  through L1 instead of staging them, with the same arithmetic).
* The uneven-M mixed workload, one segment per fit, matches the float64 oracle at
  the parity bars (1e-4 parameters, 1e-5 chi2, >= 99.9% status agreement).
* Graph replay, arena growth, empty segments, the fixed (one fit per warp)
  mapping, argument errors and the autotuner.
"""

import numpy as np
import pytest

from batchfit_b200 import accuracy as A
from batchfit_b200 import workloads as W

pytestmark = pytest.mark.gpu

PARAM_TOL, CHI2_TOL, STATUS_AGREE = 1e-4, 1e-5, 0.999
P = {"gaussian": 3, "lorentzian": 3, "pseudo_voigt": 4, "two_lorentzian": 8}


def spectra(model, n, m, seed):
    """Seeded spectra of the mixed workload's distributions on linspace(-10, 10, m)."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-10, 10, m)
    a = rng.uniform(0.5, 5.0, n)[:, None]
    c = rng.uniform(-6, 6, n)[:, None]
    w = np.exp(rng.uniform(np.log(0.1), np.log(3.0), n))[:, None]
    if model == "gaussian":
        clean = a * np.exp(-0.5 * ((x - c) / (w / 2.354820045)) ** 2)
    elif model == "lorentzian":
        clean = a / (1 + ((x - c) / (w / 2)) ** 2)
    elif model == "pseudo_voigt":
        eta = rng.uniform(0, 1, n)[:, None]
        z = (x - c) / w
        clean = a * ((1 - eta) * np.exp(-4 * np.log(2) * z * z) + eta / (1 + 4 * z * z))
    else:
        w2 = np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))[:, None]
        c2 = c + rng.uniform(0.5, 3.0, n)[:, None] * 0.5 * (w / 2 + w2)
        a2 = a * rng.uniform(0.1, 1.0, n)[:, None]
        clean = a / (1 + ((x - c) / (w / 2)) ** 2) + a2 / (1 + ((x - c2) / w2) ** 2)
    y = clean + 0.01 * a * rng.normal(size=clean.shape)
    lo, hi = W.MIXED_BOUNDS[model]
    return x.astype(np.float32), y.astype(np.float32), (np.array(lo, np.float32), np.array(hi, np.float32))


def requests(seed=11):
    """Segments of every model, M from 17 to 4099 (ragged, not multiples of 4)."""
    out = []
    shapes = [("gaussian", 33, 64), ("lorentzian", 57, 129), ("pseudo_voigt", 300, 512),
              ("two_lorentzian", 41, 1024), ("pseudo_voigt", 5, 4099), ("gaussian", 9, 2047),
              ("lorentzian", 1, 17), ("two_lorentzian", 12, 3001), ("pseudo_voigt", 70, 250)]
    for i, (model, n, m) in enumerate(shapes):
        x, y, bounds = spectra(model, n, m, seed + i)
        out.append(dict(x=x, y=y, model=model, bounds=bounds, uncertainties=(i % 2 == 0)))
    return out


def to_np(result):
    return {k: getattr(result, k).cpu().numpy() for k in result._fields}


def test_segments_equal_single_calls(bf):
    import torch

    reqs = requests()
    compared = 0
    for lanes in (8, 16, 32):
        batch = bf.fit_batch([dict(r, group_lanes=lanes) for r in reqs])
        for r, got in zip(reqs, batch):
            alone = bf.fit(torch.as_tensor(r["x"]).cuda(), torch.as_tensor(r["y"]).cuda(), r["model"], None,
                           r["bounds"], "cuda", uncertainties=r["uncertainties"], group_lanes=lanes)
            if bf.context(0).timing().group_lanes != lanes:
                continue  # the staged path widened the groups to fit shared memory
            compared += 1
            a, b = to_np(got), to_np(alone)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"{r['model']} M={r['x'].size} lanes={lanes} {k}")
    assert compared >= 20


def test_given_p0_and_mixed_policies(bf):
    import torch

    reqs = requests(seed=40)
    for i, r in enumerate(reqs):
        if i % 3 == 0:
            p0, _ = bf.guess(r["x"], r["y"], r["model"])
            r["p0"] = p0
        if i % 4 == 1:
            r["policy"] = "reference"
        r["group_lanes"] = 16
    batch = bf.fit_batch(reqs)
    for r, got in zip(reqs, batch):
        alone = bf.fit(torch.as_tensor(r["x"]).cuda(), torch.as_tensor(r["y"]).cuda(), r["model"], r.get("p0"),
                       r["bounds"], "cuda", uncertainties=r["uncertainties"], group_lanes=16,
                       policy=r.get("policy", "parity"))
        if bf.context(0).timing().group_lanes != 16:
            continue
        a, b = to_np(got), to_np(alone)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_graph_replay_and_arena_growth(bf):
    reqs = requests(seed=70)
    direct = [to_np(r) for r in bf.fit_batch(reqs, graph=False)]
    for _ in range(2):  # the first graph call captures, the second replays
        again = [to_np(r) for r in bf.fit_batch(reqs)]
        for a, b in zip(direct, again):
            for k in a:
                np.testing.assert_array_equal(a[k], b[k])
    # A larger batch grows the arena (new graph), a smaller one reuses it.
    big = requests(seed=71) + requests(seed=72) + requests(seed=73)
    got_big = [to_np(r) for r in bf.fit_batch(big)]
    ref_big = [to_np(r) for r in bf.fit_batch(big, graph=False)]
    for a, b in zip(got_big, ref_big):
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    small = [to_np(r) for r in bf.fit_batch(reqs[:2])]
    for a, b in zip(small, direct[:2]):
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_graph_enables_only_the_batch_class_types(bf):
    """The replayed graph holds one LM kernel per (model, lanes) class type and a
    batch enables only its own types: batches whose type sets change from call to
    call (one model, another, all, a subset) equal their direct launches bit for
    bit, and so does a batch past the graph's size (launched directly)."""
    reqs = requests(seed=80)
    by_model = {m: [r for r in reqs if r["model"] == m] for m in P}
    sequence = [by_model["gaussian"], by_model["two_lorentzian"], reqs, by_model["pseudo_voigt"],
                by_model["lorentzian"] + by_model["two_lorentzian"], by_model["gaussian"]]
    for batch in sequence:
        direct = [to_np(r) for r in bf.fit_batch(batch, graph=False)]
        replayed = [to_np(r) for r in bf.fit_batch(batch)]
        for a, b in zip(direct, replayed):
            for k in a:
                np.testing.assert_array_equal(a[k], b[k])
    x, y, bounds = spectra("pseudo_voigt", 40000, 64, 81)
    big = [dict(x=x, y=y, model="pseudo_voigt", bounds=bounds)] + by_model["two_lorentzian"]
    got = [to_np(r) for r in bf.fit_batch(big)]
    ref = [to_np(r) for r in bf.fit_batch(big, graph=False)]
    for a, b in zip(got, ref):
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    assert np.isin(got[0]["status"], (0, 5)).mean() > 0.9


def test_fixed_mapping_is_one_warp_per_fit(bf):
    reqs = requests(seed=90)
    fixed = bf.fit_batch(reqs, fixed_mapping=True)
    wide = bf.fit_batch([dict(r, group_lanes=32) for r in reqs])
    for a, b in zip(fixed, wide):
        a, b = to_np(a), to_np(b)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_empty_segments_and_empty_batch(bf):
    assert bf.fit_batch([]) == []
    x, y, bounds = spectra("lorentzian", 4, 64, 5)
    res = bf.fit_batch([dict(x=x, y=y[:0], model="lorentzian", bounds=bounds),
                        dict(x=x, y=y, model="lorentzian", bounds=bounds)])
    assert res[0].params.shape == (0, 3)
    alone = bf.fit_batch([dict(x=x, y=y, model="lorentzian", bounds=bounds)])
    np.testing.assert_array_equal(res[1].params.cpu().numpy(), alone[0].params.cpu().numpy())
    np.testing.assert_array_equal(res[1].status.cpu().numpy(), alone[0].status.cpu().numpy())


def test_argument_errors(bf):
    x, y, bounds = spectra("gaussian", 2, 64, 6)
    with pytest.raises(ValueError):
        bf.fit_batch([dict(x=x, y=y, model="nope")])
    xl = np.linspace(-10, 10, bf._capi.load().bf_cuda_batch_max_points() + 1).astype(np.float32)
    with pytest.raises(ValueError, match="segment 0"):
        bf.fit_batch([dict(x=xl, y=np.zeros((1, xl.size), np.float32), model="gaussian")])
    with pytest.raises(ValueError):
        bf.fit_batch([dict(x=x, y=y, model="gaussian", group_lanes=12)])


def test_mixed_uneven_stream_matches_oracle(bf, oracle):
    w = W.mixed_stream(n=1200, seed=4)
    names = W.MODEL_NAMES
    reqs = []
    for i in range(w.models.size):
        s, m = int(w.offsets[i]), int(w.counts[i])
        model = names[int(w.models[i])]
        lo, hi = W.MIXED_BOUNDS[model]
        reqs.append(dict(x=w.x[s:s + m], y=w.y[s:s + m].reshape(1, m), model=model,
                         bounds=(np.array(lo, np.float32), np.array(hi, np.float32))))
    got = bf.fit_batch(reqs)
    # Fits the float64 oracle leaves at max_iterations (100 attempts) have no
    # definite status: on this workload they are unresolved peaks (FWHM below the
    # grid spacing) that the reference's own float32 path reports as unresolved.
    # They must not converge on the GPU either.  On every other fit statuses agree
    # at the parity bar (>= 99.9%); >= 99% of all converged fits and of each
    # single-peak model's (>= 95% of the two-Lorentzian's) are within 1e-4 / 1e-5 of
    # the float64 solution or
    # float32-equivalent to it (float64 chi2 within the float32 evaluation error of
    # the oracle's); the single-peak models are plainly within 1e-4 for >= 97% (the
    # stream holds peaks narrower than its coarsest grids), and the two-Lorentzian
    # requests overlapping doublets whose parameters no float32 evaluation pins to 1e-4.
    definite = agree = chi2_ok = converged = 0
    within = {m: [0, 0, 0] for m in names}  # within, within or equivalent, converged
    equivalent = within_ref32 = within_all = 0
    for r, g in zip(reqs, got):
        lo, hi = r["bounds"]
        ref = oracle.fit("port", r["model"], r["x"], r["y"], None, lo, hi, np.float64)
        gs = g.status.cpu().numpy()
        if ref.status[0] == 1:
            assert gs[0] in (1, 5), (r["model"], r["x"].size, gs[0])
            continue
        ref32 = oracle.fit("port", r["model"], r["x"], r["y"], None, lo, hi, np.float32)
        s = A.summarize(r["model"], r["x"], r["y"], g.params.cpu().numpy(), gs, g.chi2.cpu().numpy(), ref.params,
                        ref.status, ref.chi2, PARAM_TOL, CHI2_TOL, x64=True)
        s32 = A.summarize(r["model"], r["x"], r["y"], ref32.params, ref32.status, ref32.chi2, ref.params,
                          ref.status, ref.chi2, PARAM_TOL, CHI2_TOL)
        definite += 1
        agree += s["status_agreement"]
        within_all += s["within_tol_fraction"]
        within_ref32 += s32["within_tol_fraction"]
        if ref.status[0] in (0, 5) and gs[0] == ref.status[0]:
            within[r["model"]][0] += s["within_tol_fraction"]
            within[r["model"]][1] += s["within_or_equivalent_fraction"]
            within[r["model"]][2] += 1
            equivalent += s["within_or_equivalent_fraction"]
        if ref.status[0] == 0 and gs[0] == 0:
            converged += 1
            chi2_ok += s["chi2_within_fraction"]
    assert definite >= 1150
    assert agree / definite >= STATUS_AGREE, (agree, definite)
    assert equivalent >= 0.99 * sum(v[2] for v in within.values()), (equivalent, within)
    assert within["two_lorentzian"][1] >= 0.95 * within["two_lorentzian"][2], within
    for model in ("gaussian", "lorentzian", "pseudo_voigt"):
        assert within[model][1] >= 0.99 * within[model][2], (model, within)
        assert within[model][0] >= 0.97 * within[model][2], (model, within)
    assert within_all >= within_ref32, (within_all, within_ref32, definite)
    assert chi2_ok / converged >= STATUS_AGREE, (chi2_ok, converged)


def test_mixed_group_widths_in_one_batch(bf):
    import torch

    reqs = requests(seed=120)
    for i, r in enumerate(reqs):
        r["group_lanes"] = (8, 16, 32)[i % 3]
    got = bf.fit_batch(reqs)
    for r, g in zip(reqs, got):
        alone = bf.fit(torch.as_tensor(r["x"]).cuda(), torch.as_tensor(r["y"]).cuda(), r["model"], None,
                       r["bounds"], "cuda", uncertainties=r["uncertainties"], group_lanes=r["group_lanes"])
        if bf.context(0).timing().group_lanes != r["group_lanes"]:
            continue
        a, b = to_np(g), to_np(alone)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_autotune_table(bf):
    lanes = bf.autotune()
    assert len(lanes) == 4 and all(len(row) == 8 for row in lanes)
    assert all(v in (8, 16, 32) for row in lanes for v in row)
    t = bf.context(0).get_tuning()
    assert t.tuned == 1
    assert all(t.lm_ms[m][b][w] > 0 for m in range(4) for b in range(8) for w in range(3))
    # The test requests form classes far smaller than a GPU wave, which run on whole
    # warps whatever the table says: their results are the 32-lane single calls.
    reqs = requests(seed=99)
    got = bf.fit_batch(reqs)
    import torch

    for r, g in zip(reqs, got):
        alone = bf.fit(torch.as_tensor(r["x"]).cuda(), torch.as_tensor(r["y"]).cuda(), r["model"], None,
                       r["bounds"], "cuda", uncertainties=r["uncertainties"], group_lanes=32)
        a, b = to_np(g), to_np(alone)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


@pytest.mark.parametrize("m", [1539, 6147, 10240])
def test_batch_guess_equals_reference_guess(bf, oracle, m):
    """The batch guess (x and y read in place, the shared-memory sort above
    M = 5129) equals the reference float guess: a segment fitted from p0=None gives
    the same bits as the same segment fitted from the oracle's guesses."""
    x, y = W.noisy_doublets(m, 40, seed=m)
    p0, status, _ = oracle.guess("port", "two_lorentzian", x, y, np.float32)
    ok = status == 0
    assert ok.sum() >= 10
    bounds = W.MIXED_BOUNDS["two_lorentzian"]
    bounds = (np.array(bounds[0], np.float32), np.array(bounds[1], np.float32))
    base = dict(x=x, y=y[ok], model="two_lorentzian", bounds=bounds, group_lanes=32)
    guessed, given = bf.fit_batch([base, dict(base, p0=p0[ok].astype(np.float32))])
    a, b = to_np(guessed), to_np(given)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"M={m} {k}")
