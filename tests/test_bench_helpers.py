"""Host-side helpers of bench.py (no GPU): peak lookup, percentiles, roofline work."""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from batchfit_b200 import roofline  # noqa: E402


def test_hbm_peak_has_a_source():
    gbs, source = bench.hbm_peak()
    assert gbs > 1000 and ("of measured" in source or "of fallback" in source)


def test_percentile():
    assert bench.percentile([], 50) is None
    v = list(range(1, 101))
    assert bench.percentile(v, 50) == 50 and bench.percentile(v, 99) == 99 and bench.percentile(v, 100) == 100


def test_fit_work_counts():
    w = roofline.point_work("pseudo_voigt")
    assert (w.linearize_flops, w.cost_flops, w.jacobian_flops, w.mufu_per_eval) == (52, 15, 43, 2)
    flops, mufu = roofline.fit_work("pseudo_voigt", 512, 4.91, 5.90, True)
    assert abs(flops - 512 * (4.91 * 52 + 5.90 * 15 + 43)) < 1e-6
    assert abs(mufu - 512 * 2 * (4.91 + 5.90 + 1)) < 1e-6
    assert roofline.observation_bytes(512, 4, True) == 4 * 512 + 4 * 4 + 12 + 4 * (16 + 4 + 1)
