"""Streaming-replay entry point with explicit parameters.

``run_streaming_replay_b200`` has the signature of the reference's
``run_streaming_replay`` (streaming.py:365-379) and of the CUDA backend's
``run_streaming_replay_cuda``.  Parameter objects are read by attribute name,
so the reference's own AuxiliaryParameters / ScoreParameters /
DecisionParameters / ReconstructionParameters / DitherBounds / LCG24 and the
small dataclasses below are interchangeable.
"""

from __future__ import annotations

import hashlib
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .engine import StreamingReplayResult, context, replay_result, run_frame
from .profile import RESPONSE_LUT_SHA256

LCG24_MASK = 0x00FF_FFFF


@dataclass(frozen=True)
class AuxiliaryParameters:  # x3a.py:166-179
    selected_visible_channel: int
    alpha: float
    calibration_offset: float
    alpha_one_replacement: float | None


@dataclass(frozen=True)
class ScoreParameters:  # x3a.py:224-242
    base_primary: float
    base_addend: float
    scale: float
    offset: float
    floor: float
    resolution_metric: int
    horizontal_minimum_resolution_cutoff: int


@dataclass(frozen=True)
class DecisionParameters:  # x3a.py:337-348
    sample_threshold: float
    count_limit: int
    perpendicular_radius: int


@dataclass(frozen=True)
class ReconstructionParameters:  # reconstruction.py:613-669
    resolution_metric: int
    cross_neighbor_cutoff: int
    coarse_enabled: bool
    coarse_reference: float
    coarse_slopes: tuple
    band_enabled: tuple
    band_scales: tuple
    factors_a: tuple
    factors_b: tuple
    configured_strengths: tuple
    driver_gate_primary: bool
    driver_gate_secondary: bool
    row_reconstruction_gate: int
    dither_scales: tuple


@dataclass(frozen=True)
class DitherBounds:  # dither.py:34-56
    low: float
    high: float
    low_index: int = 0
    high_index: int = 0


@dataclass
class LCG24:  # rng.py:138-172 (state owner only; draws happen on the device)
    state: int

    @classmethod
    def from_nikon_pe_initial_state(cls) -> "LCG24":
        return cls(0x3045)


def _f32(value) -> float:
    return float(np.float32(value))


def hot_path_params(auxiliary, score, decision, reconstruction, bounds) -> _lib.FxParams:
    """Pack reference-style parameter objects into fx_params (float32)."""

    if auxiliary.selected_visible_channel not in (0, 1, 2):
        raise ValueError("selected_visible_channel must be 0, 1, or 2")
    if not 1 <= decision.perpendicular_radius <= 4:
        raise ValueError("perpendicular_radius must be in [1, 4]")
    if not 0 <= decision.count_limit <= 9:
        raise ValueError("count_limit must be in [0, 9]")
    numeric = (reconstruction.coarse_reference, *reconstruction.coarse_slopes,
               *reconstruction.band_scales,
               *(v for row in reconstruction.factors_a for v in row),
               *(v for row in reconstruction.factors_b for v in row),
               *reconstruction.configured_strengths, *reconstruction.dither_scales)
    if not all(math.isfinite(float(v)) for v in numeric):
        raise ValueError("reconstruction parameters must be finite")
    c = _lib.FxParams()
    c.score_addend = _f32(score.base_addend)
    c.score_scale = _f32(score.scale)
    c.score_offset = _f32(score.offset)
    c.score_floor = _f32(score.floor)
    c.horizontal_minimum = int(score.horizontal_minimum_resolution_cutoff < score.resolution_metric)
    c.visible_channel = int(auxiliary.selected_visible_channel)
    c.decision_threshold = _f32(decision.sample_threshold)
    c.count_limit = int(decision.count_limit)
    c.radius = int(decision.perpendicular_radius)
    c.cross_neighbor = int(reconstruction.resolution_metric > reconstruction.cross_neighbor_cutoff)
    c.coarse_enabled = int(bool(reconstruction.coarse_enabled))
    c.coarse_slopes[:] = [_f32(v) for v in reconstruction.coarse_slopes]
    c.band_enabled[:] = [int(bool(v)) for v in reconstruction.band_enabled]
    c.band_scales[:] = [_f32(v) for v in reconstruction.band_scales]
    c.factors_a[:] = [_f32(v) for row in reconstruction.factors_a for v in row]
    c.factors_b[:] = [_f32(v) for row in reconstruction.factors_b for v in row]
    c.configured_strengths[:] = [_f32(v) for v in reconstruction.configured_strengths]
    c.driver_gate_primary = int(bool(reconstruction.driver_gate_primary))
    c.dither_scales[:] = [_f32(v) for v in reconstruction.dither_scales]
    c.dither_low = _f32(bounds.low)
    c.dither_high = _f32(bounds.high)
    return c


def stage_table(height: int, auxiliary, score, reconstruction, provider) -> np.ndarray:
    """Resolve the per-stage calibration the replay reads (streaming.py:109-133,
    429-443; startup.py:331-346)."""

    stages = np.zeros(height + 6, dtype=_lib.STAGE_DTYPE)
    if provider is None:
        replacement = auxiliary.alpha_one_replacement
        stages["alpha"] = np.float32(auxiliary.alpha)
        stages["offset"] = np.float32(auxiliary.calibration_offset)
        stages["replacement"] = np.float32(0.0 if replacement is None else replacement)
        stages["replacement_valid"] = 0 if replacement is None else 1
        stages["score_base"] = np.float32(score.base_primary)
        stages["coarse"] = np.float32(reconstruction.coarse_reference)
        stages["gate_secondary"] = int(bool(reconstruction.driver_gate_secondary))
        stages["row_gate"] = int(reconstruction.row_reconstruction_gate)
        return stages
    for hit in range(1, height + 7):
        cal = provider(hit)
        if getattr(cal, "stage_hit", hit) != hit:
            raise ValueError(f"stage parameter provider returned calibration for stage "
                             f"{cal.stage_hit}, expected {hit}")
        values = (cal.auxiliary_alpha, cal.calibration_offset, cal.base_primary)
        if not all(math.isfinite(float(v)) for v in values):
            raise ValueError("stage calibration contains a non-finite value")
        st = stages[hit - 1]
        st["alpha"] = np.float32(cal.auxiliary_alpha)
        st["offset"] = np.float32(cal.calibration_offset)
        st["replacement"] = np.float32(cal.base_primary)
        st["replacement_valid"] = 1
        st["score_base"] = np.float32(cal.base_primary)
        st["coarse"] = np.float32(cal.base_primary)
        st["gate_secondary"] = int(bool(cal.writer_gate_secondary))
        st["row_gate"] = int(cal.row_reconstruction_gate)
    return stages


def run_streaming_replay_b200(
    main_rgbi,
    output_rgb16,
    *,
    response,
    auxiliary_parameters,
    score_parameters,
    decision_parameters,
    reconstruction_parameters,
    dither_bounds,
    generator=None,
    stage_parameter_provider=None,
    progress=None,
    diagnostics_row=None,
    device: int = 0,
) -> StreamingReplayResult:
    """Execute the full main pass on the GPU with explicit parameters.

    ``output_rgb16`` is written only after the device pass succeeded.
    ``generator`` (an object with a ``state``) is advanced to the final state.
    ``diagnostics_row`` receives (y, score_row, score_floor, rendered_row,
    changed_row) per row; the last argument is the per-pixel changed mask
    (the device does not materialise the no-op image).
    """

    pixels = np.asarray(main_rgbi)
    output = np.asarray(output_rgb16)
    if pixels.dtype != np.dtype(np.uint16) or pixels.ndim != 3 or pixels.shape[2] != 4:
        raise ValueError("streaming main input must be uint16 HxWx4")
    height, width, _ = pixels.shape
    if height < 4:
        raise ValueError("streaming startup requires at least four main rows")
    if output.dtype != np.dtype(np.uint16) or output.shape != (height, width, 3):
        raise ValueError("streaming output must be uint16 HxWx3")
    if not output.flags.writeable:
        raise ValueError("streaming output must be writable")
    table = np.asarray(getattr(response, "table", response), dtype=np.float32)
    if hashlib.sha256(table.astype("<f4").tobytes()).hexdigest() != RESPONSE_LUT_SHA256:
        raise ValueError("the B200 path supports only the shared Nikon logarithmic response")
    params = hot_path_params(auxiliary_parameters, score_parameters, decision_parameters,
                             reconstruction_parameters, dither_bounds)
    stages = stage_table(height, auxiliary_parameters, score_parameters,
                         reconstruction_parameters, stage_parameter_provider)
    state = 0x3045 if generator is None else int(generator.state) & LCG24_MASK
    ctx = context(device)
    outcome = run_frame(ctx, pixels, params, stages, state, diagnostics_row is not None)
    result = replay_result(outcome)
    np.copyto(output, outcome.output)
    if generator is not None:
        generator.state = result.final_rng_state
    floor = np.float32(score_parameters.floor)
    if diagnostics_row is not None or progress is not None:
        for y in range(height):
            if diagnostics_row is not None:
                diagnostics_row(y, outcome.score[y], floor, outcome.output[y],
                                outcome.changed[y].astype(bool))
        if progress is not None:
            progress(height, height, result.attempted_pixels, result.written_pixels)
    return result
