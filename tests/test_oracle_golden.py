"""Pin the CPU oracle to the reference: golden vectors and reference runs.

The oracle is the checker for every GPU parity test, so it is pinned first:
  * the reference's own known answers (tests/test_engine.py:28-33,
    tests/test_core.py:20-30, the hybrid example's pinned digests);
  * results the reference produced on seeded inputs (reference_results.json,
    written by golden/make_golden.py): output digest, all counters, the
    startup receipt, diagnostics digests, prepass records and producer
    schedules.
"""

from __future__ import annotations

import struct

import numpy as np
import pytest

import cases
from _helpers import SLOW_JOBS, oracle_direct, oracle_mismatches, sha
from oracle import oracle as ox


def test_reference_table_and_rng_pins():
    """tests/test_core.py:20-30: LUT hash, normalisation bytes, first states."""

    assert ox.response_lut().shape == (65536,)
    assert struct.pack("<f", float.fromhex("0x1.fffffep-25")) == bytes.fromhex("ffff7f33")
    state, states = 0x3045, []
    for _ in range(4):
        state = (125 * state + 1) & 0xFFFFFF
        states.append(state)
    assert states == [0x1791B2, 0x8223EB, 0x8B89C0, 0x2242C1]


def test_engine_8x8_known_answer():
    """tests/test_engine.py:28-33 pins this job's digest and counters."""

    res = ox.process(*cases.engine_8x8())
    assert res.output_sha256 == "8d0992222a7523de293d69de38d560131ccf9bef2b90be9f7942406743a07941"
    assert res.attempted_pixels == 8
    assert res.written_pixels == res.changed_pixels == 2
    assert res.public_rng_advances == 26


def test_hybrid_example_pinned_digests():
    """hybrid/examples/synthetic-lama/run/diagnostics-cache/diagnostics-cache.json."""

    res = ox.process(*cases.hybrid_256())
    assert res.output_sha256 == "780257c669f8df3f3f47768dbd99ffe61354de5f3b66e1b2c8bdedd0cc0e4ad8"
    assert sha(res.score_plane.astype("<f4")) == (
        "566c3b0648d5c91566f2a4db3834d39fa9be934ab596ef4c9d188a9c8a3d9baa")
    assert sha(res.at_floor_mask) == (
        "ac7c5f191ce8f1150114da25edaa0a14ca1ba1c67a679bf980900fa56148af94")
    assert sha(res.changed_mask) == (
        "b652da2639bc8ee709d3cd026598f9acc085bc6ad464671507f8eecc150b40c5")
    assert res.startup_advances == (0, 1107, 1152, 1159, 1176, 1145)


FAST_JOBS = [n for n in cases.JOB_CASES if n not in SLOW_JOBS]


@pytest.mark.parametrize("name", FAST_JOBS)
def test_oracle_matches_reference_jobs(name, golden):
    expected = golden["jobs"][name]
    main, prepass = cases.JOB_CASES[name][0]()
    assert sha(main.astype("<u2")) == expected["input_sha256"], "input recipe drifted"
    res = ox.process(main, prepass)
    assert oracle_mismatches(expected, res) == []
    assert res.prepass_payload.hex() == expected["prepass_payload"]


@pytest.mark.slow
@pytest.mark.parametrize("name", ["native_full", "heavy_full_0"])
def test_oracle_matches_reference_full_frame(name, golden):
    """Full 5782x3946 frames (the native frame and a heavy-damage frame at
    about 5% coverage) against the reference's cpu-fast runs."""

    expected = golden["jobs"][name]
    main, prepass = cases.JOB_CASES[name][0]()
    assert sha(main.astype("<u2")) == expected["input_sha256"], "input recipe drifted"
    res = ox.process(main, prepass)
    assert oracle_mismatches(expected, res) == []


@pytest.mark.parametrize("name", sorted(cases.DIRECT_CASES))
def test_oracle_matches_reference_direct_cases(name, golden):
    expected = golden["direct"][name]
    pixels, spec = cases.direct_case(name)
    res = oracle_direct(pixels, spec)
    got = {
        "output_sha256": res.output_sha256, "attempted_pixels": res.attempted_pixels,
        "written_pixels": res.written_pixels, "public_rng_advances": res.public_rng_advances,
        "final_rng_state": res.final_rng_state, "changed_pixels": res.changed_pixels,
        "startup_attempted": list(res.startup_attempted),
        "startup_advances": list(res.startup_advances),
        "startup_final_state": res.startup_final_state,
    }
    assert got == expected


@pytest.mark.parametrize("geometry", cases.PRODUCER_CASES, ids=lambda g: f"{g[0]}x{g[1]}")
def test_oracle_producer_schedule(geometry, golden):
    h, w, seed = geometry
    expected = golden["producer"][f"{h}x{w}_seed{seed}"]
    rows = ox.producer_rows(cases.producer_pixels(h, w, seed))
    assert sha(rows["p2"].astype("<f4")) == expected["input_scale_sha256"]
    assert sha(rows["p1"].astype("<f4")) == expected["scaled_input_sha256"]
    assert sha(rows["mean_vis"].astype("<f4")) == expected["mean_visible_sha256"]
    assert sha(rows["mean_ir"].astype("<f4")) == expected["mean_infrared_sha256"]


def test_oracle_detects_a_planted_mistake():
    """A checker that cannot fail is no checker: corrupt one stage and the
    oracle's digest must move."""

    main, prepass = cases.self_test_job()
    good = ox.process(main, prepass)
    stages = good.stages.copy()
    stages["coarse"][10] = np.float32(stages["coarse"][10] + 1.0)
    bad = ox.replay(main, stages)
    assert bad.output_sha256 != good.output_sha256
