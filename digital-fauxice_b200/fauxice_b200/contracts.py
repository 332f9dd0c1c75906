"""Acquisition contracts with the reference's names, fields and messages.

Mirrors portable_digital_ice contracts.py:18-221 (RGBI16Frame,
DualRGBIAcquisition, PrepassFrameRecord) and profile.py:296-318
(ScannerModel, ProcessingMode, ProcessingJob) so a job built with either
package is accepted by the other's validation.
"""

from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from enum import Enum

import numpy as np
import numpy.typing as npt

UInt16Array = npt.NDArray[np.uint16]


class AcquisitionEpoch(str, Enum):
    PREPASS = "prepass"
    MAIN = "main"


class ScannerModel(str, Enum):
    NIKON_SUPER_COOLSCAN_5000_ED = "nikon-super-coolscan-5000-ed"


class ProcessingMode(str, Enum):
    NORMAL = "normal"


def _frozen_uint16_image(pixels: npt.ArrayLike, *, lanes: int, label: str) -> UInt16Array:
    """contracts.py:25-40: copy into a read-only C-order uint16 array."""

    array = np.asarray(pixels)
    if array.dtype != np.dtype(np.uint16):
        raise TypeError(f"{label} must have dtype uint16")
    if array.ndim != 3 or array.shape[2] != lanes:
        raise ValueError(f"{label} must have shape HxWx{lanes}")
    if array.shape[0] < 1 or array.shape[1] < 1:
        raise ValueError(f"{label} cannot have an empty dimension")
    owned = np.array(array, dtype=np.uint16, order="C", copy=True)
    owned.flags.writeable = False
    return owned


@dataclass(frozen=True)
class RGBI16Frame:
    """contracts.py:43-74: one immutable interleaved 16-bit RGBI acquisition."""

    pixels: UInt16Array
    epoch: AcquisitionEpoch
    resolution_dpi: int
    evidence_id: str

    def __post_init__(self) -> None:
        if self.resolution_dpi <= 0:
            raise ValueError("resolution_dpi must be positive")
        if not self.evidence_id.strip():
            raise ValueError("evidence_id must be non-empty")
        object.__setattr__(self, "pixels",
                           _frozen_uint16_image(self.pixels, lanes=4, label="RGBI frame"))

    @property
    def height(self) -> int:
        return int(self.pixels.shape[0])

    @property
    def width(self) -> int:
        return int(self.pixels.shape[1])

    @property
    def sha256(self) -> str:
        return hashlib.sha256(self.pixels.astype("<u2", copy=False).tobytes(order="C")).hexdigest()


@dataclass(frozen=True)
class DualRGBIAcquisition:
    """contracts.py:161-175: the required same-frame prepass/main pair."""

    prepass: RGBI16Frame
    main: RGBI16Frame
    same_frame_id: str

    def __post_init__(self) -> None:
        if _enum_value(self.prepass.epoch) != AcquisitionEpoch.PREPASS.value:
            raise ValueError("prepass frame has the wrong acquisition epoch")
        if _enum_value(self.main.epoch) != AcquisitionEpoch.MAIN.value:
            raise ValueError("main frame has the wrong acquisition epoch")
        if not self.same_frame_id.strip():
            raise ValueError("same_frame_id must be non-empty")


@dataclass(frozen=True)
class PrepassFrameRecord:
    """contracts.py:178-221: the opaque 0x40-byte record."""

    payload: bytes
    frame_index: int
    evidence_id: str

    def __post_init__(self) -> None:
        payload = bytes(self.payload)
        if len(payload) != 0x40:
            raise ValueError("prepass frame record must contain exactly 0x40 bytes")
        if self.frame_index < 0:
            raise ValueError("prepass frame index cannot be negative")
        if not self.evidence_id.strip():
            raise ValueError("prepass frame record evidence_id must be non-empty")
        object.__setattr__(self, "payload", payload)

    @property
    def sha256(self) -> str:
        return hashlib.sha256(self.payload).hexdigest()

    @property
    def observed_main_alpha(self) -> np.float32:
        return np.float32(struct.unpack_from("<f", self.payload, 0x04)[0])

    @property
    def observed_calibration_mean_r(self) -> np.float32:
        return np.float32(struct.unpack_from("<f", self.payload, 0x28)[0])

    @property
    def observed_calibration_mean_ir(self) -> np.float32:
        return np.float32(struct.unpack_from("<f", self.payload, 0x2C)[0])


@dataclass(frozen=True)
class ProcessingJob:
    """profile.py:308-318: one explicitly identified dual RGBI acquisition."""

    acquisition: DualRGBIAcquisition
    scanner_model: ScannerModel
    mode: ProcessingMode
    selector: int
    resolution_metric: int
    bit_depth: int
    focus_exposure_locked: bool


def _enum_value(value):
    return getattr(value, "value", value)


def is_processing_job(job) -> bool:
    """Accept this package's ProcessingJob or the reference's (same fields)."""

    if isinstance(job, ProcessingJob):
        return True
    return type(job).__name__ == "ProcessingJob" and all(
        hasattr(job, name)
        for name in ("acquisition", "scanner_model", "mode", "selector", "resolution_metric",
                     "bit_depth", "focus_exposure_locked")
    )


def is_dual_acquisition(acquisition) -> bool:
    if isinstance(acquisition, DualRGBIAcquisition):
        return True
    return type(acquisition).__name__ == "DualRGBIAcquisition" and all(
        hasattr(acquisition, name) for name in ("prepass", "main", "same_frame_id")
    )
