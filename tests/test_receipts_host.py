"""Parity receipts on the host: comparison figures, status and encoding.

The receipt follows the reference's evidence receipts
(evidence/cuda-frame-1-parity.json): a sample-by-sample comparison of the
RGB16 output with the reference's, the counters and the fixtures' hashes,
encoded as canonical JSON (hybrid receipts.py:322-337).
"""

from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np

import cases
from fauxice_b200 import receipts
from oracle import oracle as ox


def _result_from_oracle(res):
    startup = SimpleNamespace(attempted_per_stage=tuple(res.startup_attempted),
                              rng_advances_per_stage=tuple(res.startup_advances),
                              final_rng_state=res.startup_final_state)
    replay = SimpleNamespace(output_sha256=res.output_sha256, attempted_pixels=res.attempted_pixels,
                             written_pixels=res.written_pixels, changed_pixels=res.changed_pixels,
                             public_rng_advances=res.public_rng_advances,
                             final_rng_state=res.final_rng_state, startup=startup)
    return SimpleNamespace(output_rgb16=res.output_rgb16, replay=replay, profile_id="p")


def test_equal_outputs_pass_and_encode_canonically(tmp_path):
    main, prepass = cases.self_test_job()
    res = ox.process(main, prepass)
    doc = receipts.parity_receipt(_result_from_oracle(res), res.output_rgb16, main=main,
                                  prepass=prepass, claim="oracle against itself",
                                  elapsed_seconds=0.25)
    assert doc["status"] == "PASS"
    assert doc["mismatch_samples"] == doc["mismatch_pixels"] == 0
    assert doc["compared_rgb16_samples"] == res.output_rgb16.size
    assert doc["b200_output_sha256"] == doc["reference_output_sha256"] == res.output_sha256
    payload = receipts.canonical_receipt_bytes(doc)
    assert payload.endswith(b"\n") and b" " not in payload.split(b'"claim"')[0]
    assert json.loads(payload) == json.loads(json.dumps(doc))
    digest = receipts.write_receipt(str(tmp_path / "r.json"), doc)
    assert digest == receipts.receipt_sha256(doc)
    assert (tmp_path / "r.json").read_bytes() == payload


def test_a_planted_difference_fails_with_its_figures():
    main, prepass = cases.self_test_job()
    res = ox.process(main, prepass)
    bad = res.output_rgb16.copy()
    bad[3, 4, 1] ^= 5
    bad[7, 0, :] = 0
    figures = receipts.compare_rgb16(bad, res.output_rgb16)
    expected = np.abs(bad.astype(np.int64) - res.output_rgb16.astype(np.int64))
    assert figures["mismatch_samples"] == int((expected != 0).sum())
    assert figures["mismatch_pixels"] == int((expected != 0).any(axis=-1).sum())
    assert figures["maximum_absolute_delta"] == int(expected.max())
    assert figures["absolute_delta_sum"] == int(expected.sum())
    doc = receipts.parity_receipt(_result_from_oracle(res), bad, main=main, prepass=prepass,
                                  claim="planted")
    assert doc["status"] == "FAIL"
