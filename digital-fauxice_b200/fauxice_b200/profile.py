"""The one validated profile and the constant tables of the hot path.

Mirrors portable_digital_ice profile.py:335-456 (LS-5000, selector 8,
Normal, metric 4000): the same fail-closed validation, every float constant
given as its float32 bit pattern, and the response LUT / inverse-response
factor tables regenerated from their equations (x3a.py:111-132,
output.py:40-58) and checked against the reference's pinned SHA-256 digests.
"""

from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from functools import lru_cache

import numpy as np

from . import _lib
from .contracts import _enum_value, is_dual_acquisition, is_processing_job

RESPONSE_LUT_SHA256 = "5fd225e25719a544df9475315e3017f9b8027d593ac43e392245de59f49f3fcb"
H_FACTOR_SHA256 = "fdc378493f13916e36d3dbd9b69b714e888d7993680509df4550486db6fcf328"
L_FACTOR_SHA256 = "b7f3b1b5c0ea816ddb20196e1cf7614d364ea4e164295e0dcb78119c88ef404d"
NIKON_PE_INITIAL_STATE = 0x3045


class UnboundBehaviorError(RuntimeError):
    """A platform table did not reproduce its pinned digest."""


def f32_from_bits(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits))[0]


@lru_cache(maxsize=1)
def response_lut() -> np.ndarray:
    """float32(65535 * log2(v + 1) / 16) for v in 0..65535, hash-pinned."""

    domain = np.arange(65536, dtype=np.float64)
    table = np.asarray(65535.0 * np.log2(domain + np.float64(1.0)) / 16.0, dtype=np.float32,
                       order="C")
    if hashlib.sha256(table.astype("<f4", copy=False).tobytes()).hexdigest() != \
            RESPONSE_LUT_SHA256:
        raise UnboundBehaviorError(
            "platform logarithm does not reproduce Nikon's response LUT bit-exact")
    table.flags.writeable = False
    return table


@lru_cache(maxsize=1)
def factor_tables() -> tuple[np.ndarray, np.ndarray]:
    """The high- and low-byte inverse-response factors, hash-pinned."""

    domain = np.arange(256, dtype=np.float64)
    scale = 16.0 * np.log10(np.float64(2.0)) / 65535.0
    high = np.floor(16.0 * np.power(10.0, 256.0 * domain * scale) + 0.5).astype(np.uint32)
    low = np.floor(65536.0 * np.power(10.0, domain * scale) + 0.5).astype(np.uint32)
    digests = (hashlib.sha256(high.astype("<u4", copy=False).tobytes()).hexdigest(),
               hashlib.sha256(low.astype("<u4", copy=False).tobytes()).hexdigest())
    if digests != (H_FACTOR_SHA256, L_FACTOR_SHA256):
        raise UnboundBehaviorError(
            "platform power function did not reproduce the recovered inverse-response factor "
            "tables")
    high.flags.writeable = False
    low.flags.writeable = False
    return high, low


def dither_bounds(lut: np.ndarray, maximum_index: int = 65_535) -> tuple[float, float]:
    """dither.py:18-56: table values at the truncated 1% / 99% indices."""

    n = np.float32(maximum_index)
    low_index = min(int(np.trunc(float(np.multiply(n, np.float32(0.01))))), maximum_index)
    high_index = min(int(np.trunc(float(np.multiply(n, np.float32(0.99))))), maximum_index)
    return float(lut[low_index]), float(lut[high_index])


@dataclass(frozen=True)
class HotPathParameters:
    """Every scalar the kernels read (float32 values), in reference terms."""

    score_addend: float
    score_scale: float
    score_offset: float
    score_floor: float
    horizontal_minimum: bool
    visible_channel: int
    decision_threshold: float
    count_limit: int
    radius: int
    cross_neighbor: bool
    coarse_enabled: bool
    coarse_slopes: tuple
    band_enabled: tuple
    band_scales: tuple
    factors_a: tuple  # 9 values, [band][channel]
    factors_b: tuple
    configured_strengths: tuple
    driver_gate_primary: bool
    dither_scales: tuple
    dither_low: float
    dither_high: float

    def to_c(self) -> _lib.FxParams:
        c = _lib.FxParams()
        f = lambda v: float(np.float32(v))  # noqa: E731
        c.score_addend = f(self.score_addend)
        c.score_scale = f(self.score_scale)
        c.score_offset = f(self.score_offset)
        c.score_floor = f(self.score_floor)
        c.horizontal_minimum = int(bool(self.horizontal_minimum))
        c.visible_channel = int(self.visible_channel)
        c.decision_threshold = f(self.decision_threshold)
        c.count_limit = int(self.count_limit)
        c.radius = int(self.radius)
        c.cross_neighbor = int(bool(self.cross_neighbor))
        c.coarse_enabled = int(bool(self.coarse_enabled))
        c.coarse_slopes[:] = [f(v) for v in self.coarse_slopes]
        c.band_enabled[:] = [int(bool(v)) for v in self.band_enabled]
        c.band_scales[:] = [f(v) for v in self.band_scales]
        c.factors_a[:] = [f(v) for v in self.factors_a]
        c.factors_b[:] = [f(v) for v in self.factors_b]
        c.configured_strengths[:] = [f(v) for v in self.configured_strengths]
        c.driver_gate_primary = int(bool(self.driver_gate_primary))
        c.dither_scales[:] = [f(v) for v in self.dither_scales]
        c.dither_low = f(self.dither_low)
        c.dither_high = f(self.dither_high)
        return c


def _base_primary(payload: bytes) -> np.float32:
    """profile.py:48-55: raises when the prepass alpha is exactly one."""

    alpha = np.float32(struct.unpack_from("<f", payload, 0x04)[0])
    mean_r = np.float32(struct.unpack_from("<f", payload, 0x28)[0])
    mean_ir = np.float32(struct.unpack_from("<f", payload, 0x2C)[0])
    denominator = 1.0 - float(alpha)
    if denominator == 0.0:
        raise ValueError("prepass alpha cannot equal one")
    return np.float32((float(mean_ir) - float(alpha) * float(mean_r)) / denominator)


@dataclass(frozen=True, init=False)
class LS5000Selector8NormalProfile:
    """profile.py:335-453: the single scanner, mode and resolution contract."""

    scanner_model: str = "nikon-super-coolscan-5000-ed"
    mode: str = "normal"
    selector: int = 8
    resolution_metric: int = 4_000
    prepass_dpi: int = 285
    main_dpi: int = 4_000
    bit_depth: int = 16
    auxiliary_factor_b: float = 1.0

    @property
    def profile_id(self) -> str:
        return "nikon-ls5000-selector8-normal-metric4000"

    def validate_job(self, job) -> None:
        """Reject every scanner, mode and acquisition outside this profile."""

        if not is_processing_job(job):
            raise TypeError("processing requires a ProcessingJob")
        expected = (
            ("scanner model", job.scanner_model, self.scanner_model),
            ("mode", job.mode, self.mode),
            ("selector", job.selector, self.selector),
            ("resolution metric", job.resolution_metric, self.resolution_metric),
            ("bit depth", job.bit_depth, self.bit_depth),
        )
        for label, actual, supported in expected:
            if _enum_value(actual) != supported:
                shown = supported if label not in ("scanner model", "mode") else _enum_repr(
                    label, supported)
                raise ValueError(
                    f"unsupported {label} {actual!r}; this profile requires {shown!r}")
        if job.focus_exposure_locked is not True:
            raise ValueError("main capture must retain prepass focus and exposure")
        acquisition = job.acquisition
        if not is_dual_acquisition(acquisition):
            raise TypeError("processing requires a dual RGBI acquisition")
        if acquisition.prepass.resolution_dpi != self.prepass_dpi:
            raise ValueError(f"prepass must be captured at {self.prepass_dpi} dpi")
        if acquisition.main.resolution_dpi != self.main_dpi:
            raise ValueError(f"main frame must be captured at {self.main_dpi} dpi")
        main = acquisition.main.pixels
        if main.shape[0] < 5 or main.shape[1] < 8:
            raise ValueError("main RGBI frame must be at least 5 rows by 8 columns")
        if (main.shape[1] // 8) * 8 == 0:
            raise ValueError("main RGBI frame has no complete producer cell")

    def hot_path_parameters(self) -> HotPathParameters:
        """profile.py:404-453 constants as float32 values."""

        f = f32_from_bits
        low, high = dither_bounds(response_lut())
        return HotPathParameters(
            score_addend=f(0xC2EED000),
            score_scale=f(0xBA887952),
            score_offset=f(0x3F800000),
            score_floor=f(0x3CA3D70A),
            horizontal_minimum=550 < self.resolution_metric,
            visible_channel=0,
            decision_threshold=f(0x4740E73C),
            count_limit=8,
            radius=4,
            cross_neighbor=self.resolution_metric > 1_600,
            coarse_enabled=True,
            coarse_slopes=(f(0x3F8CCCCD),) * 3,
            band_enabled=(True, True, True),
            band_scales=(f(0x3FA00000),) * 3,
            factors_a=tuple(f(b) for b in (0x3F9AE148, 0x3F9D70A4, 0x3F90A3D7, 0x3F95C28F,
                                           0x3F91EB85, 0x3F8A3D71, 0x3F851EB8, 0x3F6E147B,
                                           0x3F7851EC)),
            factors_b=tuple(f(b) for b in (0x3F8B851F, 0x3F90A3D7, 0x3F851EB8, 0x3F8A3D71,
                                           0x3F866666, 0x3F828F5C, 0x3F75C28F, 0x3F570A3D,
                                           0x3F63D70A)),
            configured_strengths=(0.0, 0.0, 0.0),
            driver_gate_primary=True,
            dither_scales=(f(0x3C75C28F), f(0x3C75C28F), f(0x3CCCCCCD)),
            dither_low=low,
            dither_high=high,
        )

    def score_floor(self) -> np.float32:
        return np.float32(f32_from_bits(0x3CA3D70A))

    def check_prepass_record(self, payload: bytes) -> None:
        """The profile derivations raise on an alpha of exactly one."""

        _base_primary(payload)


def _enum_repr(label: str, value: str):
    from .contracts import ProcessingMode, ScannerModel

    return ScannerModel(value) if label == "scanner model" else ProcessingMode(value)


DEFAULT_PROFILE = LS5000Selector8NormalProfile()
