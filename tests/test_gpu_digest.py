"""The output SHA-256 that fx_process computes while copying the output back.

The library hashes each staged chunk as soon as it lands; the digest must
equal hashlib's SHA-256 of the returned output (little-endian uint16 bytes,
row-major), from an 8 x 8 frame (16 chunks of 24 bytes) to multi-megabyte
frames.
"""

from __future__ import annotations

import ctypes
import hashlib

import numpy as np
import pytest

import cases
from fauxice_b200 import _lib, engine
from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(8, 8), (17, 33), (130, 257), (600, 411)])
def test_library_digest_equals_hashlib(shape):
    ctx = engine.context()
    px = cases.generated(31 + shape[0], shape[0], shape[1], "native")[0]
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    for _ in range(2):  # two calls in a row: no state carried between digests
        outcome = engine.run_frame(ctx, px, params, None, NIKON_PE_INITIAL_STATE, False)
        assert outcome.digest is not None
        expected = hashlib.sha256(outcome.output.astype("<u2").tobytes()).digest()
        assert outcome.digest == expected
        assert engine.replay_result(outcome).output_sha256 == expected.hex()


def test_digest_is_refused_when_disabled():
    lib = _lib.load()
    ctx = engine.context()
    buf = (ctypes.c_uint8 * 32)()
    try:
        assert lib.fx_set_output_digest(ctx.handle, 0) == 0
        assert lib.fx_output_digest(ctx.handle, buf) != 0
    finally:
        assert lib.fx_set_output_digest(ctx.handle, 1) == 0


def test_parity_receipt_of_a_device_result(tmp_path):
    """A receipt for a B200 result against the oracle's output passes, with
    the device's runtime recorded."""

    import time

    import cases
    from _helpers import make_job
    from fauxice_b200 import receipts
    from fauxice_b200.engine import process_b200
    from oracle import oracle as ox

    main, prepass = cases.generated(71, 200, 333, "heavy")
    t0 = time.perf_counter()
    result = process_b200(make_job(main, prepass))
    elapsed = time.perf_counter() - t0
    doc = receipts.parity_receipt(result, ox.process(main, prepass).output_rgb16, main=main,
                                  prepass=prepass, claim="200x333 heavy frame against the oracle",
                                  elapsed_seconds=elapsed)
    assert doc["status"] == "PASS" and doc["mismatch_samples"] == 0
    assert doc["runtime"]["compute_capability"] == "10.0"
    assert receipts.write_receipt(str(tmp_path / "receipt.json"), doc) == receipts.receipt_sha256(doc)
