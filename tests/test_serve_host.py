"""Host logic of the serving loop (no GPU): arrival schedule and report."""

from __future__ import annotations

import numpy as np

from fauxice_b200 import _lib, serve


def test_poisson_arrivals_are_seeded_sorted_and_bounded():
    a = serve.poisson_arrivals(8.0, 30.0, seed=3)
    b = serve.poisson_arrivals(8.0, 30.0, seed=3)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0) and a.min() >= 0 and a.max() < 30.0
    assert 150 < a.size < 330  # mean 240


def test_report_percentiles_and_throughput():
    report = serve.ServeReport(wall_s=2.0, megapixels=100.0)
    for i, lat in enumerate([0.010, 0.020, 0.030, 0.040]):
        report.completions.append(serve.Completion(i, 1.0, 1.0, 1.0 + lat, _lib.FxCounters()))
    s = report.summary()
    assert s["requests"] == 4 and s["mp_per_s"] == 50.0
    assert s["p50_ms"] == 25.0
    assert s["p50_ms"] <= s["p95_ms"] <= s["p99_ms"] <= 40.0
