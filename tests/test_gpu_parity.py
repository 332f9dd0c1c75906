"""B200 parity: every output uint16, counter and diagnostics plane bit-exact.

Compared against the reference's recorded results (reference_results.json:
pure-Python process_cpu for crops up to 512x512, the numba cpu-fast backend
for full frames) and against the CPU oracle on fresh seeded frames.  All
calls go through the C ABI (libfauxice_b200.so via ctypes).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases
from _helpers import SLOW_JOBS, b200_mismatches, direct_objects, make_job, oracle_direct, sha
from fauxice_b200 import _lib, engine, streaming
from fauxice_b200.backend import b200_self_test, process
from fauxice_b200.engine import ProcessingCancelled, process_b200
from fauxice_b200.profile import DEFAULT_PROFILE, response_lut
from oracle import oracle as ox

pytestmark = pytest.mark.gpu


def test_self_test_known_answers():
    b200_self_test()


@pytest.mark.parametrize("name", [n for n in cases.JOB_CASES if n not in SLOW_JOBS])
def test_jobs_match_reference(name, golden):
    main, prepass = cases.JOB_CASES[name][0]()
    result = process_b200(make_job(main, prepass, name), export_diagnostics=True)
    assert b200_mismatches(golden["jobs"][name], result) == []


@pytest.mark.parametrize("name", sorted(SLOW_JOBS))
def test_full_frames_match_reference(name, golden):
    """Full frames (5782x3946, 3946x5782, 2892x1973, 1024x768, 4000x2700)
    against the reference's cpu-fast backend."""

    main, prepass = cases.JOB_CASES[name][0]()
    result = process_b200(make_job(main, prepass, name), export_diagnostics=True)
    assert b200_mismatches(golden["jobs"][name], result) == []


@pytest.mark.parametrize("name", sorted(cases.DIRECT_CASES))
def test_direct_cases_match_reference(name, golden):
    pixels, spec = cases.direct_case(name)
    aux, score, decision, recon = direct_objects(spec)
    lut = response_lut()
    low, high = float(lut[655]), float(lut[64879])
    out = np.empty((pixels.shape[0], pixels.shape[1], 3), np.uint16)
    gen = streaming.LCG24.from_nikon_pe_initial_state()
    rep = streaming.run_streaming_replay_b200(
        pixels, out, response=lut, auxiliary_parameters=aux, score_parameters=score,
        decision_parameters=decision, reconstruction_parameters=recon,
        dither_bounds=streaming.DitherBounds(low, high), generator=gen)
    expected = golden["direct"][name]
    got = {
        "output_sha256": rep.output_sha256, "attempted_pixels": rep.attempted_pixels,
        "written_pixels": rep.written_pixels, "public_rng_advances": rep.public_rng_advances,
        "final_rng_state": rep.final_rng_state, "changed_pixels": rep.changed_pixels,
        "startup_attempted": list(rep.startup.attempted_per_stage),
        "startup_advances": list(rep.startup.rng_advances_per_stage),
        "startup_final_state": rep.startup.final_rng_state,
    }
    assert got == expected
    assert gen.state == expected["final_rng_state"]
    assert sha(out.astype("<u2")) == expected["output_sha256"]


def test_alpha_one_without_replacement_fails_closed():
    pixels, spec = cases.direct_case("alpha_one")
    spec["aux"]["replacement"] = None
    aux, score, decision, recon = direct_objects(spec)
    lut = response_lut()
    out = np.zeros((pixels.shape[0], pixels.shape[1], 3), np.uint16)
    from fauxice_b200.profile import UnboundBehaviorError

    with pytest.raises(UnboundBehaviorError):
        streaming.run_streaming_replay_b200(
            pixels, out, response=lut, auxiliary_parameters=aux, score_parameters=score,
            decision_parameters=decision, reconstruction_parameters=recon,
            dither_bounds=streaming.DitherBounds(float(lut[655]), float(lut[64879])))
    assert not out.any()


@pytest.mark.parametrize("geometry", cases.PRODUCER_CASES, ids=lambda g: f"{g[0]}x{g[1]}")
def test_device_producer_schedule(geometry, golden):
    h, w, seed = geometry
    ctx = engine.context()
    px = cases.producer_pixels(h, w, seed)
    rows = [np.empty(h, np.float32) for _ in range(4)]
    rc = _lib.load().fx_producer_rows(ctx.handle, _lib.ptr(px), h, w, *(_lib.ptr(r) for r in rows))
    assert rc == 0
    expected = golden["producer"][f"{h}x{w}_seed{seed}"]
    assert sha(rows[0].astype("<f4")) == expected["scaled_input_sha256"]
    assert sha(rows[1].astype("<f4")) == expected["input_scale_sha256"]
    assert sha(rows[2].astype("<f4")) == expected["mean_visible_sha256"]
    assert sha(rows[3].astype("<f4")) == expected["mean_infrared_sha256"]


@pytest.mark.parametrize("seed, h, w, spec", [
    (31, 64, 96, "native"), (32, 200, 333, "native"), (33, 8, 8, "native"),
    (34, 129, 257, "heavy"), (35, 300, 41, "small"), (36, 517, 611, "heavy"),
])
def test_fresh_frames_match_oracle(seed, h, w, spec):
    main, prepass = cases.generated(seed, h, w, spec)
    result = process_b200(make_job(main, prepass), export_diagnostics=True)
    res = ox.process(main, prepass)
    assert result.replay.output_sha256 == res.output_sha256
    assert np.array_equal(result.output_rgb16, res.output_rgb16)
    assert result.replay.attempted_pixels == res.attempted_pixels
    assert result.replay.written_pixels == res.written_pixels
    assert result.replay.public_rng_advances == res.public_rng_advances
    assert result.replay.final_rng_state == res.final_rng_state
    assert result.replay.changed_pixels == res.changed_pixels
    assert result.replay.startup.rng_advances_per_stage == res.startup_advances
    assert np.array_equal(result.diagnostics.score_plane.view(np.uint32),
                          res.score_plane.view(np.uint32))
    assert np.array_equal(result.diagnostics.changed_mask, res.changed_mask)


def test_repeat_runs_are_identical():
    main, prepass = cases.generated(41, 300, 400, "heavy")
    job = make_job(main, prepass)
    first = process_b200(job)
    second = process_b200(job)
    assert first.replay == second.replay
    assert np.array_equal(first.output_rgb16, second.output_rgb16)


def test_caller_owned_output_and_cancellation():
    main, prepass = cases.self_test_job()
    job = make_job(main, prepass)
    out = np.empty((48, 64, 3), np.uint16)
    result = process_b200(job, output_rgb16=out)
    assert result.output_rgb16 is out
    untouched = np.full((48, 64, 3), 12345, np.uint16)
    calls = {"n": 0}

    def cancel_later() -> bool:
        calls["n"] += 1
        return calls["n"] >= 3

    with pytest.raises(ProcessingCancelled):
        process_b200(job, output_rgb16=untouched, cancelled=cancel_later)
    assert np.all(untouched == 12345)


def test_process_router_selects_b200():
    main, prepass = cases.engine_8x8()
    res = process(make_job(main, prepass), backend="b200")
    assert res.selection.used.value == "b200"
    assert res.result.replay.output_sha256 == (
        "8d0992222a7523de293d69de38d560131ccf9bef2b90be9f7942406743a07941")


def test_full_frame_size_independent_properties():
    """At full size: deterministic, non-attempted pixels keep their no-op
    value, and the changed mask agrees with the counter."""

    main, prepass = cases.JOB_CASES["native_full"][0]()
    result = process_b200(make_job(main, prepass), export_diagnostics=True)
    diag = result.diagnostics
    assert int(diag.changed_mask.sum()) == result.replay.changed_pixels
    assert result.replay.written_pixels >= result.replay.changed_pixels
    assert result.replay.attempted_pixels >= result.replay.written_pixels
    assert np.array_equal(diag.at_floor_mask, diag.score_plane == DEFAULT_PROFILE.score_floor())
