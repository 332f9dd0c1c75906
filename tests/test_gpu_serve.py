"""Serving loop: requests admitted as they arrive give the same results as alone.

Requests of mixed sizes arrive on a seeded Poisson schedule and overlap on
the device (continuous batching through context slots); every request's
output and counters must equal its single-frame run, and the latency report
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
    return out.cpu().numpy().view(np.uint16), ctr


def test_served_requests_match_single_frame_runs():
    ctx = engine.context()
    rng = np.random.default_rng(77)
    arrivals = serve.poisson_arrivals(200.0, 0.08, seed=5)
    assert arrivals.size >= 8
    requests = []
    for k, t in enumerate(arrivals):
        h, w = int(rng.integers(40, 420)), int(rng.integers(40, 420))
        spec = ("native", "heavy", "small")[k % 3]
        requests.append(serve.Request(float(t), cases.generated(900 + k, h, w, spec)[0]))
    report = serve.serve(ctx, requests, slots=3, keep_outputs=True)
    assert [c.index for c in report.completions] == list(range(len(requests)))
    for c in report.completions:
        out, ctr = _alone(ctx, requests[c.index].pixels)
        assert np.array_equal(c.output, out), c.index
        for f in ("attempted", "written", "public_advances", "changed", "final_state",
                  "startup_final_state"):
            assert getattr(c.counters, f) == getattr(ctr, f), (c.index, f)
        assert c.done_s >= c.admitted_s >= c.arrival_s
    summary = report.summary()
    assert summary["requests"] == len(requests)
    assert summary["p50_ms"] <= summary["p95_ms"] <= summary["p99_ms"]
