"""The continuous-batching server: requests of different models, M and N arrive
while others run, are admitted under a device-memory budget and coalesced into
mixed batches.  Each result is the one the same request gives alone, within the
parity tolerances (1e-4 parameters, 1e-5 chi2, >= 99.9% equal statuses); the
budget is never exceeded; bad requests are refused at submission.
"""

import threading
import time

import numpy as np
import pytest

from batchfit_b200 import accuracy as A
from batchfit_b200 import workloads as W

pytestmark = pytest.mark.gpu

NAMES = ("gaussian", "lorentzian", "pseudo_voigt", "two_lorentzian")


def make_requests(count, seed, n_max=600, m_range=(64, 2048)):
    """Seeded requests like the serving stream (N, M log-uniform; random model;
    half with uncertainties)."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        model = NAMES[rng.integers(4)]
        n = int(np.exp(rng.uniform(0, np.log(n_max))))
        m = int(np.exp(rng.uniform(np.log(m_range[0]), np.log(m_range[1]))))
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
            clean = a / (1 + ((x - c) / (w / 2)) ** 2) + a * rng.uniform(0.1, 1, n)[:, None] / (1 + ((x - c2) / w2) ** 2)
        y = (clean + 0.01 * a * rng.normal(size=clean.shape)).astype(np.float32)
        lo, hi = W.MIXED_BOUNDS[model]
        reqs.append(dict(x=x.astype(np.float32), y=y, model=model,
                         bounds=(np.array(lo, np.float32), np.array(hi, np.float32)),
                         uncertainties=bool(i % 2)))
    return reqs


def same_within_tolerance(req, got, ref):
    s = A.summarize(req["model"], req["x"], req["y"], got.params, got.status, got.chi2, ref.params.cpu().numpy(),
                    ref.status.cpu().numpy(), ref.chi2.cpu().numpy(), 1e-4, 1e-5)
    return s["status_agreement"], s["within_tol_fraction"], len(got.status)


def test_results_equal_alone_under_staggered_arrivals(bf):
    reqs = make_requests(60, seed=5)
    tickets = [None] * len(reqs)
    with bf.Server() as server:
        def producer():
            rng = np.random.default_rng(1)
            for i, r in enumerate(reqs):
                tickets[i] = server.submit(r["x"], r["y"], r["model"], None, r["bounds"],
                                           uncertainties=r["uncertainties"])
                time.sleep(float(rng.exponential(0.002)))

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        results = [t.result() for t in tickets]
        st = server.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["memory_in_use"] == 0
    assert st["batches"] >= 1
    agree = within = total = 0
    for r, got in zip(reqs, results):
        alone = bf.fit_batch([r])[0]
        a, w, n = same_within_tolerance(r, got, alone)
        agree += a * n
        within += w * n
        total += n
        if r["uncertainties"]:
            ok = (got.uncertainty_status == 0) & (alone.uncertainty_status.cpu().numpy() == 0)
            np.testing.assert_allclose(got.stderr[ok], alone.stderr.cpu().numpy()[ok], rtol=2e-3)
    assert agree / total >= 0.999 and within / total >= 0.999, (agree, within, total)


def test_memory_budget_queues_requests(bf):
    reqs = make_requests(24, seed=9, n_max=400, m_range=(1024, 2048))
    budget = 24 << 20
    with bf.Server(memory_budget=budget) as server:
        tickets = [server.submit(r["x"], r["y"], r["model"], None, r["bounds"], uncertainties=r["uncertainties"])
                   for r in reqs]
        results = [t.result() for t in tickets]
        st = server.stats()
    assert st["memory_budget"] == budget
    assert 0 < st["memory_peak"] <= budget
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for r, got in zip(reqs, results):
        alone = bf.fit_batch([r])[0]
        a, w, n = same_within_tolerance(r, got, alone)
        assert a >= 0.99 and w >= 0.99


def test_refused_requests(bf):
    with bf.Server(memory_budget=1 << 20) as server:
        x = np.linspace(-10, 10, 512).astype(np.float32)
        with pytest.raises(ValueError, match="budget"):
            server.submit(x, np.zeros((2000, 512), np.float32), "gaussian")
        big = np.linspace(-10, 10, 20000).astype(np.float32)
        with pytest.raises(ValueError):
            server.submit(big, np.zeros((1, big.size), np.float32), "gaussian")
        with pytest.raises(ValueError):
            server.submit(x, np.zeros((1, 511), np.float32), "gaussian")
        t = server.submit(x, np.zeros((3, 512), np.float32), "gaussian")
        res = t.result()
        assert res.status.shape == (3,)


def test_close_completes_outstanding_requests(bf):
    reqs = make_requests(12, seed=13)
    server = bf.Server()
    tickets = [server.submit(r["x"], r["y"], r["model"], None, r["bounds"]) for r in reqs]
    results = [t._result for t in tickets]
    server.close()  # waits for every request
    for r, got in zip(reqs, results):
        alone = bf.fit_batch([dict(r, uncertainties=False)])[0]
        a, w, n = same_within_tolerance(r, got, alone)
        assert a >= 0.99


def test_allocation_failure_and_cancellation_leave_the_others_intact(bf):
    """Failure handling on the host, without a GPU fault: an admission whose device
    allocation fails (injected: the next admission's allocation reports out of
    memory) fails alone with a CUDA error, a request cancelled before admission
    raises CancelledError, and every other request completes with the result it
    gives alone; the memory budget returns to zero and the server keeps serving."""
    import concurrent.futures

    reqs = make_requests(9, seed=21, n_max=300, m_range=(1024, 1024))
    last = make_requests(1, seed=22, n_max=2, m_range=(1024, 1024))[0]
    last["y"] = np.repeat(last["y"][:1], 300, axis=0)
    reqs.append(last)
    # A budget of about one request (300 x 1024 points take ~1.3 MB) admits them
    # nearly one at a time, strictly in arrival order: the last one stays queued
    # behind the others while it is cancelled.
    budget = 2 << 20
    with bf.Server(memory_budget=budget, max_in_flight=1) as server:
        server._fail_allocations(1)
        tickets = [server.submit(r["x"], r["y"], r["model"], None, r["bounds"], uncertainties=r["uncertainties"])
                   for r in reqs]
        assert tickets[-1].cancel()
        assert tickets[-1].cancel()  # idempotent
        with pytest.raises(RuntimeError, match="failed"):
            tickets[0].result()  # the first admission took the injected failure
        with pytest.raises(concurrent.futures.CancelledError):
            tickets[-1].result()
        results = [t.result() for t in tickets[1:-1]]
        assert not tickets[1].cancel()  # completed requests cannot be cancelled
        st = server.stats()
        assert st["memory_in_use"] == 0
        assert st["failed"] == 2 and st["completed"] == len(reqs)
        # Still serving after the failures.
        again = server.submit(reqs[0]["x"], reqs[0]["y"], reqs[0]["model"], None, reqs[0]["bounds"]).result()
        assert again.status.shape == (reqs[0]["y"].shape[0],)
    for r, got in zip(reqs[1:-1], results):
        alone = bf.fit_batch([r])[0]
        a, w, n = same_within_tolerance(r, got, alone)
        assert a >= 0.99 and w >= 0.99


def test_large_request_alone_equals_the_single_call(bf):
    """A request predicted to take longer than a short batch runs alone on
    bf_cuda_fit's kernels (grids for three quarters of the SMs): its results equal
    a plain fit of the same data bit for bit, with a short request served beside it."""
    big = make_requests(1, seed=21, n_max=2)[0]
    rng = np.random.default_rng(22)
    n, m = 80000, 1024
    x = np.linspace(-10, 10, m).astype(np.float32)
    a = rng.uniform(0.5, 5.0, n)[:, None]
    c = rng.uniform(-6, 6, n)[:, None]
    w = np.exp(rng.uniform(np.log(0.1), np.log(3.0), n))[:, None]
    eta = rng.uniform(0, 1, n)[:, None]
    z = (x - c) / w
    y = (a * ((1 - eta) * np.exp(-4 * np.log(2) * z * z) + eta / (1 + 4 * z * z))
         + 0.01 * a * rng.normal(size=(n, m))).astype(np.float32)
    lo, hi = W.MIXED_BOUNDS["pseudo_voigt"]
    bounds = (np.array(lo, np.float32), np.array(hi, np.float32))
    with bf.Server() as server:
        t_big = server.submit(x, y, "pseudo_voigt", None, bounds, uncertainties=True)
        t_small = server.submit(big["x"], big["y"], big["model"], None, big["bounds"], uncertainties=False)
        got, small = t_big.result(), t_small.result()
        st = server.stats()
    assert st["failed"] == 0 and st["memory_in_use"] == 0
    ref = bf.fit(x, y, "pseudo_voigt", None, bounds, "cuda", uncertainties=True)
    for k in ("params", "status", "iterations", "chi2", "covariance", "stderr", "uncertainty_status"):
        want = getattr(ref, k)
        want = want.cpu().numpy() if hasattr(want, "cpu") else np.asarray(want)
        np.testing.assert_array_equal(np.asarray(getattr(got, k)), want, err_msg=k)
    alone = bf.fit_batch([dict(big, uncertainties=False)])[0]
    a_, w_, _ = same_within_tolerance(big, small, alone)
    assert a_ == 1.0 and w_ >= 0.99
    # With initial values given (no guess kernel): again the single call's results.
    p0 = np.where(np.isfinite(got.params), got.params, 1.0).astype(np.float32)
    with bf.Server() as server:
        got0 = server.submit(x, y, "pseudo_voigt", p0, bounds, uncertainties=False).result()
    ref0 = bf.fit(x, y, "pseudo_voigt", p0, bounds, "cuda")
    for k in ("params", "status", "iterations", "chi2"):
        want = getattr(ref0, k)
        want = want.cpu().numpy() if hasattr(want, "cpu") else np.asarray(want)
        np.testing.assert_array_equal(np.asarray(getattr(got0, k)), want, err_msg=k)
