"""Parity receipts: what one processed frame was compared with, and how.

The reference keeps one JSON receipt per validated frame and backend
(evidence/cuda-frame-1-parity.json:1-50, schema
"portable-digital-ice-cuda-parity-receipt-v1"): the geometry, a sample-by-
sample comparison of the RGB16 output with the CPU reference's (mismatching
samples and pixels, largest and summed absolute difference), the output
SHA-256, the replay counters, the startup receipt, the input fixtures'
SHA-256 and the runtime that produced it.  :func:`parity_receipt` builds the
same document for this backend's result, and :func:`canonical_receipt_bytes`
encodes it the way the reference's receipts are encoded (sorted keys, no
whitespace, ASCII, no NaN; hybrid receipts.py:322-337).

The reference's receipts also carry hashes of its private validation
pipeline (source manifests, private receipts, gate checks); those describe
files that are not shipped and have no counterpart here.
"""

from __future__ import annotations

import hashlib
import json
import platform
from typing import Any, Mapping

import numpy as np

SCHEMA = "portable-digital-ice-b200-parity-receipt-v1"


def _sha256(array: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes(order="C")).hexdigest()


def compare_rgb16(candidate: np.ndarray, reference: np.ndarray) -> dict[str, Any]:
    """Sample-by-sample comparison of two H x W x 3 uint16 outputs."""

    a = np.asarray(candidate)
    b = np.asarray(reference)
    if a.shape != b.shape or a.dtype != np.uint16 or b.dtype != np.uint16:
        raise ValueError(f"outputs differ in shape or type: {a.shape} {a.dtype} vs "
                         f"{b.shape} {b.dtype}")
    delta = np.abs(a.astype(np.int32) - b.astype(np.int32))
    mismatch = delta != 0
    return {
        "geometry_hwc": list(a.shape),
        "compared_rgb16_samples": int(a.size),
        "mismatch_samples": int(mismatch.sum()),
        "mismatch_pixels": int(mismatch.any(axis=-1).sum()),
        "maximum_absolute_delta": int(delta.max()) if delta.size else 0,
        "absolute_delta_sum": int(delta.sum(dtype=np.int64)),
    }


def runtime_description(device: int = 0) -> dict[str, Any]:
    """The GPU, driver and runtime versions that produced a result."""

    out: dict[str, Any] = {"python": platform.python_version(), "numpy": np.__version__,
                           "machine": platform.machine(), "os": platform.system()}
    try:
        import torch

        if torch.cuda.is_available():
            props = torch.cuda.get_device_properties(device)
            out["gpu"] = props.name
            out["compute_capability"] = f"{props.major}.{props.minor}"
            out["multiprocessors"] = props.multi_processor_count
            out["cuda_runtime_version"] = torch.version.cuda
        try:
            import ctypes

            version = ctypes.c_int()
            libcuda = ctypes.CDLL("libcuda.so.1")
            if libcuda.cuDriverGetVersion(ctypes.byref(version)) == 0:
                out["driver_version"] = version.value
        except OSError:
            pass
    except ImportError:
        pass
    from . import _lib

    try:
        out["library_abi"] = int(_lib.load().fx_version())
    except OSError:
        out["library_abi"] = None
    out["build_flags"] = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
    return out


def parity_receipt(result, reference_output: np.ndarray, *, main: np.ndarray,
                   prepass: np.ndarray, claim: str, elapsed_seconds: float | None = None,
                   stage_timings: Mapping[str, float] | None = None,
                   device: int = 0) -> dict[str, Any]:
    """The receipt of one ProcessingResult compared with a reference output.

    ``status`` is PASS exactly when every RGB16 sample is equal.
    """

    comparison = compare_rgb16(result.output_rgb16, reference_output)
    rep = result.replay
    reference_sha = _sha256(np.asarray(reference_output).astype("<u2", copy=False))
    status = "PASS" if comparison["mismatch_samples"] == 0 else "FAIL"
    document: dict[str, Any] = {
        "schema": SCHEMA,
        "status": status,
        "claim": claim,
        **comparison,
        "b200_output_sha256": rep.output_sha256,
        "reference_output_sha256": reference_sha,
        "attempted_pixels": rep.attempted_pixels,
        "written_pixels": rep.written_pixels,
        "changed_pixels": rep.changed_pixels,
        "public_rng_advances": rep.public_rng_advances,
        "final_rng_state": rep.final_rng_state,
        "startup_attempted_per_stage": list(rep.startup.attempted_per_stage),
        "startup_rng_advances_per_stage": list(rep.startup.rng_advances_per_stage),
        "startup_final_rng_state": rep.startup.final_rng_state,
        "main_fixture_sha256": _sha256(np.asarray(main).astype("<u2", copy=False)),
        "prepass_fixture_sha256": _sha256(np.asarray(prepass).astype("<u2", copy=False)),
        "profile_id": result.profile_id,
        "runtime": runtime_description(device),
    }
    if elapsed_seconds is not None:
        document["runtime"]["elapsed_seconds"] = round(float(elapsed_seconds), 6)
    if stage_timings:
        document["runtime"]["stage_seconds"] = {k: round(float(v), 6)
                                                for k, v in stage_timings.items()}
    return document


def canonical_receipt_bytes(document: object) -> bytes:
    """The receipt's only accepted encoding: sorted keys, compact, ASCII."""

    return (json.dumps(document, allow_nan=False, ensure_ascii=True, separators=(",", ":"),
                       sort_keys=True).encode("utf-8") + b"\n")


def receipt_sha256(document: object) -> str:
    return hashlib.sha256(canonical_receipt_bytes(document)).hexdigest()


def write_receipt(path: str, document: Mapping[str, Any]) -> str:
    """Write the canonical bytes; returns their SHA-256."""

    payload = canonical_receipt_bytes(document)
    with open(path, "wb") as handle:
        handle.write(payload)
    return hashlib.sha256(payload).hexdigest()


__all__ = ["SCHEMA", "compare_rgb16", "runtime_description", "parity_receipt",
           "canonical_receipt_bytes", "receipt_sha256", "write_receipt"]
