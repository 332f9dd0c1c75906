"""Both stencil tile heights are bit-exact, and the autotuner's cache works.

The analysis stencil is compiled for 8-row tiles (four blocks per SM, the
default) and 16-row tiles (two blocks per SM).  The choice may change only
the time: every golden job, direct case and full frame must match the
reference's recorded results with 16-row tiles too.  The batching autotuner
stores its choice as JSON keyed by device and frame shapes and reuses it.
"""

from __future__ import annotations

import contextlib
import json

import numpy as np
import pytest

import cases
from _helpers import b200_mismatches, direct_objects, make_job, sha
from fauxice_b200 import _lib, batch, engine, streaming
from fauxice_b200.engine import process_b200
from fauxice_b200.profile import response_lut

pytestmark = pytest.mark.gpu

JOBS = [n for n in cases.JOB_CASES if n.startswith(("engine", "hybrid", "self_test", "diag",
                                                    "multi_band", "tile_", "gen_"))]
JOBS += ["small_crop_512", "batch_3", "batch_2", "native_full", "heavy_full_0"]


@contextlib.contextmanager
def _tile(rows: int):
    ctx = engine.context()
    assert _lib.load().fx_set_stencil_tile(ctx.handle, rows) == 0
    try:
        yield ctx
    finally:
        assert _lib.load().fx_set_stencil_tile(ctx.handle, 0) == 0


@pytest.mark.parametrize("name", JOBS)
def test_sixteen_row_tiles_match_reference(name, golden):
    main, prepass = cases.JOB_CASES[name][0]()
    with _tile(16):
        result = process_b200(make_job(main, prepass, name), export_diagnostics=True)
    assert b200_mismatches(golden["jobs"][name], result) == []


@pytest.mark.parametrize("name", sorted(cases.DIRECT_CASES))
def test_sixteen_row_tiles_direct_cases(name, golden):
    pixels, spec = cases.direct_case(name)
    aux, score, decision, recon = direct_objects(spec)
    lut = response_lut()
    out = np.empty((pixels.shape[0], pixels.shape[1], 3), np.uint16)
    with _tile(16):
        rep = streaming.run_streaming_replay_b200(
            pixels, out, response=lut, auxiliary_parameters=aux, score_parameters=score,
            decision_parameters=decision, reconstruction_parameters=recon,
            dither_bounds=streaming.DitherBounds(float(lut[655]), float(lut[64879])),
            generator=streaming.LCG24.from_nikon_pe_initial_state())
    expected = golden["direct"][name]
    assert rep.output_sha256 == expected["output_sha256"]
    assert rep.final_rng_state == expected["final_rng_state"]


def test_tile_knob_rejects_other_heights():
    ctx = engine.context()
    assert _lib.load().fx_set_stencil_tile(ctx.handle, 12) == 1


def test_autotune_measures_then_reuses_its_choice(tmp_path, golden):
    import torch

    ctx = engine.context()
    frames = [cases.generated(61, 300, 257, "heavy")[0], cases.JOB_CASES["batch_3"][0]()[0],
              cases.generated(62, 517, 611, "native")[0]]
    d_in = [torch.from_numpy(np.ascontiguousarray(f).view(np.int16)).to("cuda") for f in frames]
    outs = [torch.empty((f.shape[0], f.shape[1], 3), dtype=torch.int16, device="cuda")
            for f in frames]
    jobs = [batch.DeviceFrame(d.data_ptr(), f.shape[0], f.shape[1], o.data_ptr())
            for f, d, o in zip(frames, d_in, outs)]
    path = str(tmp_path / "tuning.json")
    try:
        entry, cached = batch.autotune(ctx, jobs, candidates=(1, 2), waves=(0,), tiles=(8, 16),
                                       cache_path=path)
        assert not cached
        assert entry["stencil_tile"] in (8, 16) and entry["slots"] in (1, 2)
        assert len(entry["timings_ms"]) == 4
        stored = json.load(open(path))
        assert list(stored.values()) == [entry]
        again, cached = batch.autotune(ctx, jobs, cache_path=path)
        assert cached and again == entry
        # every tile height gives the same outputs
        results = []
        for rows in (8, 16):
            batch.set_stencil_tile(ctx, rows)
            batch.run_device_batch(ctx, jobs, slots=2)
            results.append([o.cpu().numpy().copy() for o in outs])
        for a, b in zip(*results):
            assert np.array_equal(a, b)
        assert sha(results[1][1].view(np.uint16)) == golden["jobs"]["batch_3"]["output_sha256"]
    finally:
        batch.set_stencil_tile(ctx, 0)
        batch.set_walk_wave(ctx, 0)
