"""Batched processing: every frame's result is the same in the mix as alone.

Frames of uneven sizes run concurrently in separate context slots
(fx_submit_device / fx_submit through fauxice_b200.batch).  Each output and
counter set must equal the frame's single-frame run, and the frames that
have reference results must match those.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases
from _helpers import b200_mismatches, make_job, sha
from fauxice_b200 import _lib, batch, engine
from fauxice_b200.engine import process_b200
from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE

pytestmark = pytest.mark.gpu

COUNTER_FIELDS = ("attempted", "written", "public_advances", "changed", "final_state",
                  "startup_final_state", "rng_dependent")


def _counters(c: _lib.FxCounters) -> tuple:
    return (tuple(getattr(c, f) for f in COUNTER_FIELDS) + tuple(c.startup_attempted)
            + tuple(c.startup_advances))


def _device_frames():
    frames = [cases.generated(41, 300, 257, "heavy")[0], cases.generated(42, 64, 96)[0],
              cases.JOB_CASES["batch_3"][0]()[0], cases.generated(43, 517, 611, "native")[0],
              cases.generated(44, 128, 2000, "heavy")[0], cases.generated(45, 9, 17)[0]]
    return [np.ascontiguousarray(f) for f in frames]


def test_device_batch_matches_single_frame_runs(golden):
    import torch

    ctx = engine.context()
    lib = _lib.load()
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    frames = _device_frames()
    d_in = [torch.from_numpy(f.view(np.int16)).to("cuda") for f in frames]
    alone_out, alone_ctr = [], []
    for f, d in zip(frames, d_in):
        h, w = f.shape[:2]
        out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
        ctr = _lib.FxCounters()
        torch.cuda.synchronize()
        rc = lib.fx_process_device(ctx.handle, ctypes.c_void_p(d.data_ptr()), h, w,
                                   ctypes.byref(params), None, 0x3045,
                                   ctypes.c_void_p(out.data_ptr()), None, None, None,
                                   ctypes.byref(ctr))
        assert rc == 0, ctx._error(ctx.handle)
        alone_out.append(out.cpu().numpy().view(np.uint16))
        alone_ctr.append(_counters(ctr))
    outs = [torch.full((f.shape[0], f.shape[1], 3), -1, dtype=torch.int16, device="cuda")
            for f in frames]
    torch.cuda.synchronize()
    jobs = [batch.DeviceFrame(d.data_ptr(), f.shape[0], f.shape[1], o.data_ptr())
            for f, d, o in zip(frames, d_in, outs)]
    # rounds in a row: slots and arenas are reused; the launch priority of
    # the chain and the walk changes only the order blocks are dispatched in
    try:
        for slots, priority in ((3, True), (6, True), (4, False)):
            batch.set_launch_priority(ctx, priority)
            counters = batch.run_device_batch(ctx, jobs, slots=slots)
            for k in range(len(frames)):
                got = outs[k].cpu().numpy().view(np.uint16)
                assert np.array_equal(got, alone_out[k]), (slots, priority, k)
                assert _counters(counters[k]) == alone_ctr[k], (slots, priority, k)
    finally:
        batch.set_launch_priority(ctx, True)
    expected = golden["jobs"]["batch_3"]
    assert sha(alone_out[2]) == expected["output_sha256"]


def test_host_batch_matches_reference_results(golden):
    names = ["self_test_48x64", "tile_edge", "gen_6_130x70", "diagnostics_30x40", "hybrid_256"]
    jobs = [make_job(*cases.JOB_CASES[n][0](), n) for n in names]
    results = batch.process_batch(jobs, slots=3, export_diagnostics=True)
    for name, job, result in zip(names, jobs, results):
        assert b200_mismatches(golden["jobs"][name], result) == [], name
        alone = process_b200(job)
        assert alone.replay == result.replay, name
        assert np.array_equal(alone.output_rgb16, result.output_rgb16), name


def test_batch_refuses_invalid_jobs_before_any_work():
    main, prepass = cases.engine_8x8()
    good = make_job(main, prepass)
    bad = make_job(main[:4], prepass)
    with pytest.raises(ValueError, match="at least 5 rows by 8 columns"):
        batch.process_batch([good, bad])


def test_reserved_slots_do_not_grow():
    """After fx_reserve_frames, frames within the bounds allocate no device
    memory (the free device memory stays the same)."""

    ctx = engine.context()
    lib = _lib.load()
    batch.set_slots(ctx, 2)
    batch.reserve_frames(ctx, 300, 280)
    free0, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.fx_mem_info(ctx.handle, ctypes.byref(free0), ctypes.byref(total)) == 0
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    for k, (h, w) in enumerate(((300, 280), (120, 97), (299, 13), (41, 280))):
        px = cases.generated(500 + k, h, w, "native")[0]
        engine.run_frame(ctx, px, params, None, NIKON_PE_INITIAL_STATE, False)
    free1 = ctypes.c_size_t()
    assert lib.fx_mem_info(ctx.handle, ctypes.byref(free1), ctypes.byref(total)) == 0
    assert free1.value == free0.value
    with pytest.raises(Exception):
        batch.reserve_frames(ctx, 0, 10)
