"""The writer's rare paths, forced and checked bit for bit.

On ordinary frames the speculative walk never misses its windows and the
RNG-dependent channel list never overflows, so the exact fallbacks behind
them would go untested.  Two test knobs of the C ABI drive them on purpose
(fx_set_walk_window narrows the windows, fx_set_list_capacity shrinks the
list); neither may change a result.  The frames come from the golden set, so
every run is compared with the reference's own recorded output
(reference_results.json, the reference's cpu-fast backend for these sizes).

Also here: the one-warp serial walk (fx_set_parallel_walk 0), a narrow walk
wave (fx_set_walk_wave 148), the settled-phase packing of the window walk
(two candidates per lane), cancellation of a request in flight (fx_cancel)
and result delivery through fx_fetch.
"""

from __future__ import annotations

import contextlib
import ctypes
import functools

import numpy as np
import pytest

import cases
from _helpers import job_mismatches, make_job, sha
from fauxice_b200 import _lib, batch, engine
from fauxice_b200.engine import ProcessingCancelled, process_b200
from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=3)
def _frame(name: str) -> np.ndarray:
    main, _ = cases.JOB_CASES[name][0]()
    main = np.ascontiguousarray(main)
    main.setflags(write=False)
    return main


@contextlib.contextmanager
def _knobs(ctx, *, window=None, capacity=None, parallel=None, wave=None):
    lib = _lib.load()
    try:
        if window is not None:
            assert lib.fx_set_walk_window(ctx.handle, window) == 0
        if capacity is not None:
            assert lib.fx_set_list_capacity(ctx.handle, capacity) == 0
        if parallel is not None:
            assert lib.fx_set_parallel_walk(ctx.handle, parallel) == 0
        if wave is not None:
            assert lib.fx_set_walk_wave(ctx.handle, wave) == 0
        yield
    finally:
        assert lib.fx_set_walk_window(ctx.handle, 4.5) == 0
        assert lib.fx_set_list_capacity(ctx.handle, 0) == 0
        assert lib.fx_set_parallel_walk(ctx.handle, 1) == 0
        assert lib.fx_set_walk_wave(ctx.handle, 0) == 0


def _run(ctx, name: str) -> engine.FrameOutcome:
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    return engine.run_frame(ctx, _frame(name), params, None, NIKON_PE_INITIAL_STATE, True)


def _mismatches(golden, name: str, outcome: engine.FrameOutcome) -> list[str]:
    rep = engine.replay_result(outcome)
    diag = engine.make_diagnostics(outcome, DEFAULT_PROFILE.score_floor())
    return job_mismatches(
        golden["jobs"][name], output_sha256=rep.output_sha256, attempted=rep.attempted_pixels,
        written=rep.written_pixels, advances=rep.public_rng_advances,
        final_state=rep.final_rng_state, changed=rep.changed_pixels,
        startup_attempted=rep.startup.attempted_per_stage,
        startup_advances=rep.startup.rng_advances_per_stage,
        startup_final_state=rep.startup.final_rng_state, score=diag.score_plane,
        at_floor=diag.at_floor_mask, changed_mask=diag.changed_mask)


def test_walk_window_misses_fall_back_to_the_exact_walk(golden):
    """Windows of 0 sigma (16 candidates each side): most entry counts land
    outside, and each such segment is walked exactly."""

    ctx = engine.context()
    with _knobs(ctx, window=0.0):
        outcome = _run(ctx, "batch_3")
    assert outcome.counters.walk_fallbacks > 0
    assert _mismatches(golden, "batch_3", outcome) == []


def test_walk_window_misses_on_a_full_frame(golden):
    ctx = engine.context()
    with _knobs(ctx, window=1.0):
        outcome = _run(ctx, "heavy_full_0")
    assert outcome.counters.walk_fallbacks > 0
    assert _mismatches(golden, "heavy_full_0", outcome) == []


def test_list_overflow_reruns_fx_process(golden):
    ctx = engine.context()
    with _knobs(ctx, capacity=4096):
        outcome = _run(ctx, "batch_3")
    assert outcome.counters.rng_dependent > 4096  # the first pass overflowed
    assert outcome.counters.capacity_reruns == 1
    assert _mismatches(golden, "batch_3", outcome) == []


def test_list_overflow_reruns_fx_submit(golden):
    ctx = engine.context()
    main, prepass = cases.JOB_CASES["batch_3"][0]()
    job = make_job(main, prepass, "batch_3")
    with _knobs(ctx, capacity=4096):
        results = batch.process_batch([job, job], slots=2, export_diagnostics=True)
    for result in results:
        assert result.replay.output_sha256 == golden["jobs"]["batch_3"]["output_sha256"]
        assert result.replay.final_rng_state == golden["jobs"]["batch_3"]["final_rng_state"]
        assert (sha(result.diagnostics.changed_mask)
                == golden["jobs"]["batch_3"]["changed_mask_sha256"])


def _device_input(name: str):
    import torch

    px = _frame(name)
    return px, torch.from_numpy(px.view(np.int16).copy()).to("cuda")


def test_list_overflow_reruns_fx_submit_device(golden):
    import torch

    ctx = engine.context()
    px, d_in = _device_input("batch_3")
    h, w = px.shape[:2]
    outs = [torch.full((h, w, 3), -1, dtype=torch.int16, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    frames = [batch.DeviceFrame(d_in.data_ptr(), h, w, o.data_ptr()) for o in outs]
    with _knobs(ctx, capacity=4096):
        counters = batch.run_device_batch(ctx, frames, slots=2)
    expected = golden["jobs"]["batch_3"]
    for out, ctr in zip(outs, counters):
        assert ctr.rng_dependent > 4096
        assert ctr.capacity_reruns == 1
        assert sha(out.cpu().numpy().view(np.uint16)) == expected["output_sha256"]
        assert ctr.final_state == expected["final_rng_state"]
        assert ctr.public_advances == expected["public_rng_advances"]


def test_list_overflow_reruns_fx_process_device(golden):
    import torch

    ctx = engine.context()
    lib = _lib.load()
    px, d_in = _device_input("batch_3")
    h, w = px.shape[:2]
    out = torch.full((h, w, 3), -1, dtype=torch.int16, device="cuda")
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    ctr = _lib.FxCounters()
    torch.cuda.synchronize()
    with _knobs(ctx, capacity=4096):
        rc = lib.fx_process_device(ctx.handle, ctypes.c_void_p(d_in.data_ptr()), h, w,
                                   ctypes.byref(params), None, NIKON_PE_INITIAL_STATE,
                                   ctypes.c_void_p(out.data_ptr()), None, None, None,
                                   ctypes.byref(ctr))
    assert rc == 0, ctx._error(ctx.handle)
    expected = golden["jobs"]["batch_3"]
    assert ctr.rng_dependent > 4096
    assert ctr.capacity_reruns == 1
    assert sha(out.cpu().numpy().view(np.uint16)) == expected["output_sha256"]
    assert ctr.final_state == expected["final_rng_state"]


def test_a_context_that_overflowed_keeps_the_longer_list(golden):
    """Heavy damage lists more RNG-dependent channels than the default list
    holds (half the sites).  On a fresh context the first pass reruns with a
    longer list and the context keeps that length per site, so the next heavy
    frame runs once (and fx_pass_bytes grows by the longer list); through
    fx_process and through fx_submit_device, each on its own fresh context.
    Every result equals the reference's."""

    import torch

    from fauxice_b200.profile import factor_tables, response_lut

    high, low = factor_tables()
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    px = _frame("heavy_full_0")
    h, w = px.shape[:2]
    expected = golden["jobs"]["heavy_full_0"]
    lib = _lib.load()
    fresh = _lib.Context(0, lut=response_lut(), high=high, low=low)
    try:
        before, after = ctypes.c_int64(), ctypes.c_int64()
        assert lib.fx_pass_bytes(fresh.handle, h, w, ctypes.byref(before)) == 0
        assert before.value == lib.fx_frame_bytes(h, w)
        first = engine.run_frame(fresh, px, params, None, NIKON_PE_INITIAL_STATE, True)
        second = engine.run_frame(fresh, px, params, None, NIKON_PE_INITIAL_STATE, True)
        assert lib.fx_pass_bytes(fresh.handle, h, w, ctypes.byref(after)) == 0
        assert after.value > before.value
    finally:
        fresh.close()
    assert first.counters.rng_dependent > (6 * w + h * w) // 2
    assert [first.counters.capacity_reruns, second.counters.capacity_reruns] == [1, 0]
    for outcome in (first, second):
        assert _mismatches(golden, "heavy_full_0", outcome) == []

    fresh = _lib.Context(0, lut=response_lut(), high=high, low=low)
    try:
        d_in = torch.from_numpy(px.view(np.int16).copy()).to("cuda")
        outs = [torch.full((h, w, 3), -1, dtype=torch.int16, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()
        reruns = []
        for out in outs:  # one slot: the second request finds the longer list
            frame = batch.DeviceFrame(d_in.data_ptr(), h, w, out.data_ptr())
            reruns += [c.capacity_reruns for c in batch.run_device_batch(fresh, [frame], slots=1)]
    finally:
        fresh.close()
    assert reruns == [1, 0]
    for out in outs:
        assert sha(out.cpu().numpy().view(np.uint16)) == expected["output_sha256"]


def test_one_warp_serial_walk(golden):
    ctx = engine.context()
    with _knobs(ctx, parallel=0):
        outcome = _run(ctx, "batch_3")
    assert outcome.counters.walk_candidates == 0  # no speculative windows ran
    assert _mismatches(golden, "batch_3", outcome) == []


def test_narrow_walk_wave_on_a_full_frame(golden):
    ctx = engine.context()
    with _knobs(ctx, wave=148):
        outcome = _run(ctx, "native_full")
    assert _mismatches(golden, "native_full", outcome) == []


def test_settled_phase_packs_two_candidates_per_lane(golden):
    """Segments whose survivors settle between 129 and 256 walk two
    candidates per lane in at most four warps; the counter proves the path
    ran, and the digests prove it kept every result."""

    ctx = engine.context()
    outcome = _run(ctx, "native_full")
    assert outcome.counters.walk_packed_segments > 0
    assert _mismatches(golden, "native_full", outcome) == []
    with _knobs(ctx, window=8.0):  # wider windows: more candidates settle late
        wide = _run(ctx, "native_full")
    assert wide.counters.walk_packed_segments > 0
    assert _mismatches(golden, "native_full", wide) == []


def _submit(ctx, px, out=None, score=None, changed=None) -> int:
    lib = _lib.load()
    h, w = px.shape[:2]
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    frame = _lib.FxFrame(main_rgbi=px.ctypes.data, height=h, width=w,
                         params=ctypes.pointer(params), stages=None,
                         rng_state=NIKON_PE_INITIAL_STATE,
                         rgb_out=out.ctypes.data if out is not None else None,
                         score_out=score.ctypes.data if score is not None else None,
                         changed_out=changed.ctypes.data if changed is not None else None)
    ticket = ctypes.c_int64()
    status = lib.fx_submit(ctx.handle, ctypes.byref(frame), ctypes.byref(ticket))
    assert status == 0, ctx._error(ctx.handle)
    return ticket.value


def test_cancel_stops_a_host_request_and_the_slot_recovers(golden):
    """fx_cancel right after fx_submit: the frame's 182 MB upload is still
    on the stream, so the first stage gate sees the cancel word.  The
    caller's buffer stays untouched and the next request on the same slot
    is exact."""

    ctx = engine.context()
    lib = _lib.load()
    batch.set_slots(ctx, 1)
    px = _frame("native_full")
    h, w = px.shape[:2]
    out = np.full((h, w, 3), 12345, np.uint16)
    with ctx.lock:
        ticket = _submit(ctx, px, out)
        assert lib.fx_cancel(ctx.handle, ticket) == 0
        counters = _lib.FxCounters()
        status = lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters))
    assert status == 13  # FX_ERR_CANCELLED
    assert np.all(out == 12345)
    with ctx.lock:
        assert lib.fx_cancel(ctx.handle, ticket) == 1  # the ticket is gone
        ticket = _submit(ctx, px, out)
        assert lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters)) == 0
    assert sha(out) == golden["jobs"]["native_full"]["output_sha256"]
    assert counters.final_state == golden["jobs"]["native_full"]["final_rng_state"]


def test_cancel_of_a_device_request_is_all_or_nothing(golden):
    """A device-buffer request cancelled at once either stops (its output
    buffer untouched) or had already finished (its output exact)."""

    import torch

    ctx = engine.context()
    lib = _lib.load()
    px, d_in = _device_input("native_full")
    h, w = px.shape[:2]
    out = torch.full((h, w, 3), 12345, dtype=torch.int16, device="cuda")
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    torch.cuda.synchronize()
    ticket = ctypes.c_int64()
    with ctx.lock:
        status = lib.fx_submit_device(ctx.handle, ctypes.c_void_p(d_in.data_ptr()), h, w,
                                      ctypes.byref(params), None, NIKON_PE_INITIAL_STATE,
                                      ctypes.c_void_p(out.data_ptr()), None, None,
                                      ctypes.byref(ticket))
        assert status == 0, ctx._error(ctx.handle)
        assert lib.fx_cancel(ctx.handle, ticket.value) == 0
        status = lib.fx_wait(ctx.handle, ticket.value, -1, None)
    got = out.cpu().numpy()
    if status == 13:
        assert np.all(got == 12345)
    else:
        assert status == 0
        assert sha(got.view(np.uint16)) == golden["jobs"]["native_full"]["output_sha256"]


def test_process_b200_cancelled_during_the_pass_leaves_output_untouched():
    """The callback answers False at the three phase boundaries before the
    pass and True from its first poll during the pass."""

    main, prepass = cases.JOB_CASES["native_full"][0]()
    job = make_job(main, prepass)
    out = np.full((main.shape[0], main.shape[1], 3), 4321, np.uint16)
    calls = {"n": 0}

    def cancel_during_pass() -> bool:
        calls["n"] += 1
        return calls["n"] >= 4

    with pytest.raises(ProcessingCancelled):
        process_b200(job, output_rgb16=out, cancelled=cancel_during_pass)
    assert calls["n"] == 4
    assert np.all(out == 4321)


def test_process_b200_with_a_callback_that_never_cancels(golden):
    main, prepass = cases.JOB_CASES["batch_3"][0]()
    result = process_b200(make_job(main, prepass), cancelled=lambda: False,
                          export_diagnostics=True)
    expected = golden["jobs"]["batch_3"]
    assert result.replay.output_sha256 == expected["output_sha256"]
    assert sha(result.diagnostics.score_plane.astype("<f4")) == expected["score_plane_sha256"]
    assert sha(result.diagnostics.changed_mask) == expected["changed_mask_sha256"]


def test_fetch_delivers_staged_results(golden):
    """A frame submitted without output buffers keeps its results staged;
    fx_fetch delivers them, with the at-floor mask built from the score."""

    ctx = engine.context()
    lib = _lib.load()
    px = _frame("batch_3")
    h, w = px.shape[:2]
    out = np.empty((h, w, 3), np.uint16)
    score = np.empty((h, w), np.float32)
    at_floor = np.empty((h, w), np.uint8)
    changed = np.empty((h, w), np.uint8)
    counters = _lib.FxCounters()
    with ctx.lock:
        ticket = _submit(ctx, px)
        rc = lib.fx_fetch(ctx.handle, ticket, -1, _lib.ptr(out), ctypes.byref(counters),
                          _lib.ptr(score), _lib.ptr(at_floor), _lib.ptr(changed))
    assert rc == 0, ctx._error(ctx.handle)
    expected = golden["jobs"]["batch_3"]
    assert sha(out) == expected["output_sha256"]
    assert sha(score.astype("<f4")) == expected["score_plane_sha256"]
    assert sha(at_floor.astype(bool)) == expected["at_floor_sha256"]
    assert sha(changed.astype(bool)) == expected["changed_mask_sha256"]
    assert counters.final_state == expected["final_rng_state"]
    # a request that staged no score plane cannot fetch one
    with ctx.lock:
        ticket = _submit(ctx, px, out)
        assert lib.fx_fetch(ctx.handle, ticket, -1, None, None, _lib.ptr(score), None,
                            None) == 1
        assert lib.fx_wait(ctx.handle, ticket, -1, None) == 0
