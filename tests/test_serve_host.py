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


def test_slot_model_reuses_the_smallest_fitting_buffers():
    model = serve.SlotModel(2)
    assert model.choose(100) == ("new", 100)
    model.take("new", 100)
    assert model.choose(300) == ("new", 300)
    model.take("new", 300)
    assert model.allocated == 400 and model.empty == 0
    assert model.choose(50) is None  # both slots busy
    model.give_back(300)
    model.give_back(100)
    assert model.choose(50) == ("reuse", 100)
    assert model.choose(200) == ("reuse", 300)
    assert model.choose(400) is None  # no slot holds it and none is empty
    model.take("reuse", 100)
    assert model.free_sizes == [300] and model.allocated == 400
