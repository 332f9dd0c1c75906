"""Fail-closed backend selection with the B200 backend added.

Mirrors portable_digital_ice backend.py:34-445.  ``process(job,
backend="b200")`` runs the B200 path after a per-process self-test; any
other backend name is delegated to the reference package when it is
importable (it is not needed for "b200").  ``auto`` prefers B200 and falls
through to the reference's own AUTO chain, reporting every reason.

The self-test is a known-answer test: the reference's synthetic self-test
job (backend.py:60-87, rebuilt here from the same recipe) must reproduce,
bit for bit, the output digest, all five replay counters, the startup
receipt and the three diagnostics planes that the reference's pure-Python
``process_cpu`` produces for it.  Those digests are pinned below, so the
self-test needs no CPU implementation of the path at run time.
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass
from enum import Enum

import numpy as np

from .contracts import (AcquisitionEpoch, DualRGBIAcquisition, ProcessingJob, ProcessingMode,
                        RGBI16Frame, ScannerModel)
from .engine import B200BackendUnavailable, ProcessingResult, process_b200
from .profile import DEFAULT_PROFILE


class ComputeBackend(str, Enum):
    AUTO = "auto"
    CPU = "cpu"
    CPU_FAST = "cpu-fast"
    CUDA = "cuda"
    METAL = "metal"
    B200 = "b200"


@dataclass(frozen=True)
class BackendSelection:
    requested: ComputeBackend
    used: ComputeBackend
    reason: str


@dataclass(frozen=True)
class BackendProcessingResult:
    result: ProcessingResult
    selection: BackendSelection


# Known answers for the synthetic self-test job, produced by the reference's
# process_cpu(job, export_diagnostics=True).
SELF_TEST_EXPECTED = {
    "output_sha256": "b608033bed3db085e5e323dc1422c5b9818b4746c2d04bb0b719ab4a645bca57",
    "attempted_pixels": 2815,
    "written_pixels": 2234,
    "public_rng_advances": 11488,
    "final_rng_state": 5841630,
    "changed_pixels": 2233,
    "startup_attempted": (50, 50, 54, 54, 62, 62),
    "startup_advances": (0, 241, 254, 254, 268, 268),
    "startup_final_state": 7905086,
    "score_plane_sha256": "f5b81ad2bf96d18ed52690ae0f188f2d42f1446242f2b0e933d4316aed9888da",
    "at_floor_sha256": "093cd716bef430e8d22ddad08f0d89b71f6ebd0136f4857398daa213a30fbe6d",
    "changed_mask_sha256": "d59cb5005f50925b00be6e478f18319c12934dbdd0d398ef825d075c5d7e0057",
}

_SELF_TEST_CACHE: dict[str, str | None] = {}


def synthetic_self_test_job() -> ProcessingJob:
    """The reference's self-test acquisition (backend.py:60-87)."""

    rng = np.random.default_rng(20260716)
    height, width = 48, 64
    main = rng.integers(20000, 60000, size=(height, width, 4), dtype=np.uint16)
    main[18:26, 30:39, 3] = rng.integers(200, 2000, size=(8, 9), dtype=np.uint16)
    main[0:2, 0:6, 3] = 500
    main[-2:, -6:, 3] = 700
    main[3, width - 3, 3] = 900
    prepass = rng.integers(20000, 60000, size=(24, 32, 4), dtype=np.uint16)
    prepass[10:14, 12:17, 3] = 300
    acquisition = DualRGBIAcquisition(
        prepass=RGBI16Frame(prepass, AcquisitionEpoch.PREPASS, 285, "selftest-prepass"),
        main=RGBI16Frame(main, AcquisitionEpoch.MAIN, 4000, "selftest-main"),
        same_frame_id="b200-backend-self-test",
    )
    return ProcessingJob(
        acquisition=acquisition,
        scanner_model=ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED,
        mode=ProcessingMode.NORMAL,
        selector=8,
        resolution_metric=4000,
        bit_depth=16,
        focus_exposure_locked=True,
    )


def self_test_failures(result: ProcessingResult, expected: dict = SELF_TEST_EXPECTED) -> list[str]:
    """Compare a result with the pinned known answers (cf. backend.py:90-141)."""

    failures = []
    replay = result.replay
    if replay.output_sha256 != expected["output_sha256"]:
        failures.append(f"output hash mismatch expected={expected['output_sha256']} "
                        f"b200={replay.output_sha256}")
    actual_digest = hashlib.sha256(result.output_rgb16.astype("<u2").tobytes()).hexdigest()
    if actual_digest != expected["output_sha256"]:
        failures.append("output sample mismatch")
    for field in ("attempted_pixels", "written_pixels", "public_rng_advances", "final_rng_state",
                  "changed_pixels"):
        if getattr(replay, field) != expected[field]:
            failures.append(f"{field} mismatch expected={expected[field]} "
                            f"b200={getattr(replay, field)}")
    startup = replay.startup
    if (tuple(startup.attempted_per_stage) != tuple(expected["startup_attempted"])
            or tuple(startup.rng_advances_per_stage) != tuple(expected["startup_advances"])
            or startup.final_rng_state != expected["startup_final_state"]):
        failures.append("startup receipt mismatch")
    diag = result.diagnostics
    if diag is None:
        failures.append("diagnostics planes missing from self-test run")
    else:
        checks = (
            ("score plane", diag.score_plane.astype("<f4"), "score_plane_sha256"),
            ("at-floor mask", diag.at_floor_mask, "at_floor_sha256"),
            ("changed mask", diag.changed_mask, "changed_mask_sha256"),
        )
        for label, array, key in checks:
            if hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest() != expected[key]:
                failures.append(f"{label} mismatch")
        if diag.score_floor.view(np.uint32) != DEFAULT_PROFILE.score_floor().view(np.uint32):
            failures.append("score floor mismatch")
    return failures


def b200_self_test() -> None:
    """Prove B200 bit parity on the synthetic job or raise.

    The (successful or failed) outcome is cached per process; a failure
    reason is re-raised on later calls.
    """

    cached = _SELF_TEST_CACHE.get("outcome", "unset")
    if cached is None:
        return
    if cached != "unset":
        raise B200BackendUnavailable(str(cached))
    try:
        result = process_b200(synthetic_self_test_job(), export_diagnostics=True)
        failures = self_test_failures(result)
        if failures:
            reason = "B200 self-test failed parity: " + "; ".join(failures)
            _SELF_TEST_CACHE["outcome"] = reason
            raise B200BackendUnavailable(reason)
    except Exception as error:
        if _SELF_TEST_CACHE.get("outcome", "unset") == "unset":
            _SELF_TEST_CACHE["outcome"] = f"B200 self-test raised: {error!r}"
        raise
    _SELF_TEST_CACHE["outcome"] = None


def _reference():
    try:
        import portable_digital_ice
    except Exception as error:  # pragma: no cover - depends on the environment
        raise RuntimeError(f"the portable_digital_ice package is not importable: {error}") from error
    return portable_digital_ice


def process(
    job,
    *,
    backend: ComputeBackend | str = ComputeBackend.AUTO,
    output_rgb16=None,
    progress=None,
    cancelled=None,
    export_diagnostics: bool = False,
):
    """Process one job on the requested backend with fail-closed semantics."""

    DEFAULT_PROFILE.validate_job(job)
    requested = ComputeBackend(getattr(backend, "value", backend))
    if requested is ComputeBackend.B200:
        b200_self_test()
        result = process_b200(job, output_rgb16=output_rgb16, progress=progress,
                              cancelled=cancelled, export_diagnostics=export_diagnostics)
        return BackendProcessingResult(
            result, BackendSelection(requested, ComputeBackend.B200,
                                     "explicit B200 request; self-test passed byte parity"))
    if requested is ComputeBackend.AUTO:
        try:
            b200_self_test()
        except Exception as b200_error:
            reference = _reference()
            delegated = reference.process(job, backend="auto", output_rgb16=output_rgb16,
                                          progress=progress, cancelled=cancelled,
                                          export_diagnostics=export_diagnostics)
            selection = delegated.selection
            return BackendProcessingResult(
                delegated.result,
                BackendSelection(requested, ComputeBackend(selection.used.value),
                                 f"B200 unavailable ({b200_error}); {selection.reason}"))
        result = process_b200(job, output_rgb16=output_rgb16, progress=progress,
                              cancelled=cancelled, export_diagnostics=export_diagnostics)
        return BackendProcessingResult(
            result, BackendSelection(requested, ComputeBackend.B200,
                                     "startup self-test passed byte parity"))
    reference = _reference()
    delegated = reference.process(job, backend=requested.value, output_rgb16=output_rgb16,
                                  progress=progress, cancelled=cancelled,
                                  export_diagnostics=export_diagnostics)
    return BackendProcessingResult(
        delegated.result,
        BackendSelection(requested, ComputeBackend(delegated.selection.used.value),
                         delegated.selection.reason))
