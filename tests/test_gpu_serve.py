"""Serving loop: requests admitted as they arrive give the same results as alone.

Requests of mixed sizes arrive on a seeded Poisson schedule and overlap on
the device (continuous batching through context slots); every request's
output and counters must equal its single-frame run, whether admission is
bounded by slots or by a tight device-memory budget, and the latency report
must cover every request.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases
from fauxice_b200 import _lib, engine, serve
from fauxice_b200.profile import DEFAULT_PROFILE

pytestmark = pytest.mark.gpu

FIELDS = ("attempted", "written", "public_advances", "changed", "final_state",
          "startup_final_state")


def _alone(ctx, px):
    import torch

    lib = _lib.load()
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    h, w = px.shape[:2]
    d_in = torch.from_numpy(np.ascontiguousarray(px).view(np.int16)).to("cuda")
    out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
    ctr = _lib.FxCounters()
    torch.cuda.synchronize()
    rc = lib.fx_process_device(ctx.handle, ctypes.c_void_p(d_in.data_ptr()), h, w,
                               ctypes.byref(params), None, 0x3045, ctypes.c_void_p(out.data_ptr()),
                               None, None, None, ctypes.byref(ctr))
    assert rc == 0
    return out, ctr


def _requests(seed: int, rate: float, window: float):
    rng = np.random.default_rng(77 + seed)
    arrivals = serve.poisson_arrivals(rate, window, seed=5 + seed)
    requests = []
    for k, t in enumerate(arrivals):
        h, w = int(rng.integers(40, 420)), int(rng.integers(40, 420))
        spec = ("native", "heavy", "small")[k % 3]
        requests.append(serve.Request(float(t), cases.generated(900 + k, h, w, spec)[0]))
    return requests


def _check(ctx, requests, report):
    assert [c.index for c in report.completions] == list(range(len(requests)))
    for c in report.completions:
        out, ctr = _alone(ctx, requests[c.index].pixels)
        assert np.array_equal(c.output, out.cpu().numpy().view(np.uint16)), c.index
        for f in FIELDS:
            assert getattr(c.counters, f) == getattr(ctr, f), (c.index, f)
        assert c.done_s >= c.admitted_s >= c.arrival_s


def test_served_requests_match_single_frame_runs():
    ctx = engine.context()
    requests = _requests(0, 200.0, 0.08)
    assert len(requests) >= 8
    report = serve.serve(ctx, requests, max_slots=3, keep_outputs=True)
    _check(ctx, requests, report)
    summary = report.summary()
    assert summary["requests"] == len(requests)
    assert summary["p50_ms"] <= summary["p95_ms"] <= summary["p99_ms"]
    assert summary["max_in_flight"] <= 3


def test_admission_waits_for_memory_and_verifies_on_the_device():
    """A budget that holds about two of the largest requests: the loop still
    serves every request, never exceeds the budget, and the on-device check
    against each frame's single-frame output finds no difference."""

    ctx = engine.context()
    requests = _requests(1, 400.0, 0.05)
    assert len(requests) >= 8
    for r in requests:
        r.expected, _ = _alone(ctx, r.pixels)
    largest = max(serve.frame_bytes(*r.pixels.shape[:2]) + 14 * r.pixels.shape[0]
                  * r.pixels.shape[1] for r in requests)
    budget = 2 * largest + largest // 2
    report = serve.serve(ctx, requests, max_slots=8, budget_bytes=budget, keep_outputs=True)
    _check(ctx, requests, report)
    summary = report.summary()
    assert summary["peak_device_bytes"] <= budget
    assert summary["verified"] == len(requests)
    assert summary["bit_exact"] is True


def test_an_oversized_request_is_refused_up_front():
    ctx = engine.context()
    requests = _requests(2, 400.0, 0.05)
    assert requests
    with pytest.raises(MemoryError):
        serve.serve(ctx, requests, budget_bytes=1 << 20)
