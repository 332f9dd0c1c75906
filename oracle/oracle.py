"""ctypes front end of the CPU oracle (fx_oracle.c).

TEST INFRASTRUCTURE ONLY.  The tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the parity checker.  The
B200 product never imports it.

It restates the reference orchestration ``_run_supported_job``
(portable_digital_ice engine.py:110-267): validate, prepass reduction,
content-derived producer schedule, stage table, then the streaming replay
with startup, serial writer, emit, counters and diagnostics.  The response
LUT and the inverse-response factor tables are regenerated here with the
reference's numpy formulas (x3a.py:111-132, output.py:40-58) and checked
against the reference's pinned SHA-256 values before use.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import struct
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfx_oracle.so")

# Pinned digests (x3a.py:26-28, output.py:16-17).
RESPONSE_LUT_SHA256 = "5fd225e25719a544df9475315e3017f9b8027d593ac43e392245de59f49f3fcb"
H_FACTOR_SHA256 = "fdc378493f13916e36d3dbd9b69b714e888d7993680509df4550486db6fcf328"
L_FACTOR_SHA256 = "b7f3b1b5c0ea816ddb20196e1cf7614d364ea4e164295e0dcb78119c88ef404d"

NIKON_PE_INITIAL_STATE = 0x3045  # rng.py:11
PROFILE_ID = "nikon-ls5000-selector8-normal-metric4000"  # profile.py:73-74

STATUS_MESSAGES = {
    1: "invalid argument",
    2: "out of memory",
    3: "auxiliary score input must be a finite HxW plane",
    4: "work RGB must be finite",
    5: "combiner inputs must be finite",
    6: "dither inputs must be finite",
    7: "X3A setter scale cannot equal one",
    8: "stage calibration contains a non-finite value",
    9: "alpha==1 requires the runtime-configured auxiliary replacement",
    10: "unsupported geometry",
}


class OracleError(RuntimeError):
    def __init__(self, code: int, where: str) -> None:
        super().__init__(f"{where}: {STATUS_MESSAGES.get(code, code)} (status {code})")
        self.code = code


def f32_from_bits(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def response_lut() -> np.ndarray:
    """x3a.py:111-132: float32(65535*log2(v+1)/16) in binary64, hash-pinned."""

    domain = np.arange(65536, dtype=np.float64)
    table = np.asarray(65535.0 * np.log2(domain + np.float64(1.0)) / 16.0, dtype=np.float32)
    if hashlib.sha256(table.astype("<f4").tobytes()).hexdigest() != RESPONSE_LUT_SHA256:
        raise RuntimeError("platform log2 does not reproduce the response LUT")
    return table


def factor_tables() -> tuple[np.ndarray, np.ndarray]:
    """output.py:40-58: the two uint32[256] inverse-response factor tables."""

    domain = np.arange(256, dtype=np.float64)
    scale = 16.0 * np.log10(np.float64(2.0)) / 65535.0
    high = np.floor(16.0 * np.power(10.0, 256.0 * domain * scale) + 0.5).astype(np.uint32)
    low = np.floor(65536.0 * np.power(10.0, domain * scale) + 0.5).astype(np.uint32)
    if (
        hashlib.sha256(high.astype("<u4").tobytes()).hexdigest() != H_FACTOR_SHA256
        or hashlib.sha256(low.astype("<u4").tobytes()).hexdigest() != L_FACTOR_SHA256
    ):
        raise RuntimeError("platform power does not reproduce the factor tables")
    return high, low


def dither_bounds(lut: np.ndarray) -> tuple[float, float]:
    """dither.py:18-56 with maximum_index 65535: truncated 1%/99% indices."""

    n = np.float32(65535)
    low_index = min(int(np.trunc(float(np.multiply(n, np.float32(0.01))))), 65535)
    high_index = min(int(np.trunc(float(np.multiply(n, np.float32(0.99))))), 65535)
    return float(lut[low_index]), float(lut[high_index])


# --------------------------------------------------------------------------
# ctypes mirrors of the C structs
# --------------------------------------------------------------------------


class OxStage(ctypes.Structure):
    _fields_ = [
        ("alpha", ctypes.c_float),
        ("offset", ctypes.c_float),
        ("replacement", ctypes.c_float),
        ("replacement_valid", ctypes.c_int32),
        ("score_base", ctypes.c_float),
        ("coarse", ctypes.c_float),
        ("gate_secondary", ctypes.c_int32),
        ("row_gate", ctypes.c_int32),
    ]


STAGE_DTYPE = np.dtype(
    [
        ("alpha", "<f4"),
        ("offset", "<f4"),
        ("replacement", "<f4"),
        ("replacement_valid", "<i4"),
        ("score_base", "<f4"),
        ("coarse", "<f4"),
        ("gate_secondary", "<i4"),
        ("row_gate", "<i4"),
    ]
)


class OxParams(ctypes.Structure):
    _fields_ = [
        ("score_addend", ctypes.c_float),
        ("score_scale", ctypes.c_float),
        ("score_offset", ctypes.c_float),
        ("score_floor", ctypes.c_float),
        ("horizontal_minimum", ctypes.c_int32),
        ("visible_channel", ctypes.c_int32),
        ("decision_threshold", ctypes.c_float),
        ("count_limit", ctypes.c_int32),
        ("radius", ctypes.c_int32),
        ("cross_neighbor", ctypes.c_int32),
        ("coarse_enabled", ctypes.c_int32),
        ("coarse_slopes", ctypes.c_float * 3),
        ("band_enabled", ctypes.c_int32 * 3),
        ("band_scales", ctypes.c_float * 3),
        ("factors_a", ctypes.c_float * 9),
        ("factors_b", ctypes.c_float * 9),
        ("configured_strengths", ctypes.c_float * 3),
        ("driver_gate_primary", ctypes.c_int32),
        ("dither_scales", ctypes.c_float * 3),
        ("dither_low", ctypes.c_float),
        ("dither_high", ctypes.c_float),
    ]


class OxCounters(ctypes.Structure):
    _fields_ = [
        ("attempted", ctypes.c_int64),
        ("written", ctypes.c_int64),
        ("public_advances", ctypes.c_int64),
        ("changed", ctypes.c_int64),
        ("final_state", ctypes.c_uint32),
        ("startup_final_state", ctypes.c_uint32),
        ("startup_attempted", ctypes.c_int64 * 6),
        ("startup_advances", ctypes.c_int64 * 6),
    ]


_LIB = None


def build() -> str:
    """Compile fx_oracle.c with its Makefile (idempotent)."""

    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "fx_oracle.c")
        ):
            build()
        handle = ctypes.CDLL(_LIB_PATH)
        p = ctypes.c_void_p
        handle.ox_replay.argtypes = [p, ctypes.c_int, ctypes.c_int, p, p, p, ctypes.c_uint32,
                                     p, p, p, p, p, p, ctypes.c_int]
        handle.ox_replay.restype = ctypes.c_int
        handle.ox_prepass.argtypes = [p, ctypes.c_int, ctypes.c_int, p, p, p, p]
        handle.ox_prepass.restype = ctypes.c_int
        handle.ox_producer.argtypes = [p, ctypes.c_int, ctypes.c_int, p, p, p, p, p, p, p, p, p]
        handle.ox_producer.restype = ctypes.c_int
        handle.ox_stage_table.argtypes = [ctypes.c_int, p, p, p, p, ctypes.c_float, p]
        handle.ox_stage_table.restype = ctypes.c_int
        for name, cls in (("ox_sizeof_params", OxParams), ("ox_sizeof_stage", OxStage),
                          ("ox_sizeof_counters", OxCounters)):
            fn = getattr(handle, name)
            fn.restype = ctypes.c_int
            if fn() != ctypes.sizeof(cls):
                raise RuntimeError(f"oracle struct layout mismatch for {cls.__name__}")
        if STAGE_DTYPE.itemsize != ctypes.sizeof(OxStage):
            raise RuntimeError("oracle stage dtype mismatch")
        _LIB = handle
    return _LIB


def _ptr(array: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(array.ctypes.data)


# --------------------------------------------------------------------------
# Profile (profile.py:335-453)
# --------------------------------------------------------------------------


@dataclass
class Params:
    """Every constant the hot path reads, as float32 values (profile.py)."""

    score_addend: float = f32_from_bits(0xC2EED000)
    score_scale: float = f32_from_bits(0xBA887952)
    score_offset: float = f32_from_bits(0x3F800000)
    score_floor: float = f32_from_bits(0x3CA3D70A)
    horizontal_minimum: bool = True  # cutoff 550 < metric 4000
    visible_channel: int = 0
    decision_threshold: float = f32_from_bits(0x4740E73C)
    count_limit: int = 8
    radius: int = 4
    cross_neighbor: bool = True  # metric 4000 > cutoff 1600
    coarse_enabled: bool = True
    coarse_slopes: tuple = (f32_from_bits(0x3F8CCCCD),) * 3
    band_enabled: tuple = (True, True, True)
    band_scales: tuple = (f32_from_bits(0x3FA00000),) * 3
    factors_a: tuple = tuple(
        f32_from_bits(b)
        for b in (0x3F9AE148, 0x3F9D70A4, 0x3F90A3D7, 0x3F95C28F, 0x3F91EB85, 0x3F8A3D71,
                  0x3F851EB8, 0x3F6E147B, 0x3F7851EC)
    )
    factors_b: tuple = tuple(
        f32_from_bits(b)
        for b in (0x3F8B851F, 0x3F90A3D7, 0x3F851EB8, 0x3F8A3D71, 0x3F866666, 0x3F828F5C,
                  0x3F75C28F, 0x3F570A3D, 0x3F63D70A)
    )
    configured_strengths: tuple = (0.0, 0.0, 0.0)
    driver_gate_primary: bool = True
    dither_scales: tuple = (f32_from_bits(0x3C75C28F), f32_from_bits(0x3C75C28F),
                            f32_from_bits(0x3CCCCCCD))
    dither_low: float | None = None
    dither_high: float | None = None

    def to_c(self, lut: np.ndarray) -> OxParams:
        low, high = dither_bounds(lut)
        c = OxParams()
        c.score_addend = self.score_addend
        c.score_scale = self.score_scale
        c.score_offset = self.score_offset
        c.score_floor = self.score_floor
        c.horizontal_minimum = int(self.horizontal_minimum)
        c.visible_channel = self.visible_channel
        c.decision_threshold = self.decision_threshold
        c.count_limit = self.count_limit
        c.radius = self.radius
        c.cross_neighbor = int(self.cross_neighbor)
        c.coarse_enabled = int(self.coarse_enabled)
        c.coarse_slopes[:] = list(self.coarse_slopes)
        c.band_enabled[:] = [int(v) for v in self.band_enabled]
        c.band_scales[:] = list(self.band_scales)
        c.factors_a[:] = list(self.factors_a)
        c.factors_b[:] = list(self.factors_b)
        c.configured_strengths[:] = list(self.configured_strengths)
        c.driver_gate_primary = int(self.driver_gate_primary)
        c.dither_scales[:] = list(self.dither_scales)
        c.dither_low = low if self.dither_low is None else self.dither_low
        c.dither_high = high if self.dither_high is None else self.dither_high
        return c


@dataclass
class OracleResult:
    output_rgb16: np.ndarray
    output_sha256: str
    attempted_pixels: int
    written_pixels: int
    public_rng_advances: int
    final_rng_state: int
    changed_pixels: int
    startup_attempted: tuple
    startup_advances: tuple
    startup_final_state: int
    score_plane: np.ndarray | None = None
    at_floor_mask: np.ndarray | None = None
    changed_mask: np.ndarray | None = None
    prepass_payload: bytes | None = None
    stages: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


_TABLES: dict = {}


def tables():
    if not _TABLES:
        _TABLES["lut"] = response_lut()
        _TABLES["hi"], _TABLES["lo"] = factor_tables()
    return _TABLES["lut"], _TABLES["hi"], _TABLES["lo"]


def prepass_reduce(prepass: np.ndarray) -> tuple[bytes, int, int]:
    """prepass.py:96-236 via ox_prepass; returns (payload, valid, tiles)."""

    lut, _, _ = tables()
    px = np.ascontiguousarray(prepass, dtype=np.uint16)
    payload = (ctypes.c_uint8 * 64)()
    valid = ctypes.c_int64()
    tiles = ctypes.c_int64()
    rc = lib().ox_prepass(_ptr(px), px.shape[0], px.shape[1], _ptr(lut), ctypes.byref(payload),
                          ctypes.byref(valid), ctypes.byref(tiles))
    if rc:
        raise OracleError(rc, "prepass")
    return bytes(payload), valid.value, tiles.value


def producer_rows(main: np.ndarray) -> dict[str, np.ndarray]:
    """producer_parameters.py:266-495 via ox_producer."""

    lut, _, _ = tables()
    px = np.ascontiguousarray(main, dtype=np.uint16)
    h = px.shape[0]
    out = {
        "p1": np.empty(h, np.float32),
        "p2": np.empty(h, np.float32),
        "mean_vis": np.empty(h, np.float32),
        "mean_ir": np.empty(h, np.float32),
        "cum_vis": np.empty(h, np.float64),
        "cum_ir": np.empty(h, np.float64),
        "cum_w": np.empty(h, np.float64),
        "accepted": np.empty(h, np.uint32),
    }
    rc = lib().ox_producer(_ptr(px), h, px.shape[1], _ptr(lut), _ptr(out["p1"]), _ptr(out["p2"]),
                           _ptr(out["mean_vis"]), _ptr(out["mean_ir"]), _ptr(out["cum_vis"]),
                           _ptr(out["cum_ir"]), _ptr(out["cum_w"]), _ptr(out["accepted"]))
    if rc:
        raise OracleError(rc, "producer")
    return out


def stage_table(rows: dict[str, np.ndarray], factor_b: float = 1.0) -> np.ndarray:
    """stage_parameters.py:93-197 + producer_parameters.py:498-541."""

    h = rows["p1"].shape[0]
    stages = np.zeros(h + 6, dtype=STAGE_DTYPE)
    rc = lib().ox_stage_table(h, _ptr(rows["p1"]), _ptr(rows["p2"]), _ptr(rows["mean_vis"]),
                              _ptr(rows["mean_ir"]), ctypes.c_float(factor_b), _ptr(stages))
    if rc:
        raise OracleError(rc, "stage table")
    return stages


def constant_stage_table(
    height: int,
    *,
    alpha: float,
    offset: float,
    replacement: float | None,
    score_base: float,
    coarse: float,
    gate_secondary: bool,
    row_gate: int,
) -> np.ndarray:
    """Stage table for a replay without a stage provider (streaming.py:109-111)."""

    stages = np.zeros(height + 6, dtype=STAGE_DTYPE)
    stages["alpha"] = np.float32(alpha)
    stages["offset"] = np.float32(offset)
    stages["replacement"] = np.float32(0.0 if replacement is None else replacement)
    stages["replacement_valid"] = 0 if replacement is None else 1
    stages["score_base"] = np.float32(score_base)
    stages["coarse"] = np.float32(coarse)
    stages["gate_secondary"] = int(bool(gate_secondary))
    stages["row_gate"] = int(row_gate)
    return stages


def replay(
    main: np.ndarray,
    stages: np.ndarray,
    params: Params | None = None,
    *,
    rng_state: int = NIKON_PE_INITIAL_STATE,
    threads: int = 0,
    diagnostics: bool = True,
) -> OracleResult:
    """streaming.py:365-552 via ox_replay."""

    lut, hi, lo = tables()
    prm = (params or Params()).to_c(lut)
    px = np.ascontiguousarray(main, dtype=np.uint16)
    h, w = px.shape[:2]
    if stages.dtype != STAGE_DTYPE or stages.shape != (h + 6,):
        raise ValueError("stage table must hold h+6 entries")
    stages = np.ascontiguousarray(stages)
    out = np.empty((h, w, 3), np.uint16)
    score = np.empty((h, w), np.float32) if diagnostics else None
    changed = np.empty((h, w), np.uint8) if diagnostics else None
    ctr = OxCounters()
    rc = lib().ox_replay(
        _ptr(px), h, w, _ptr(lut), ctypes.byref(prm), _ptr(stages), ctypes.c_uint32(rng_state),
        _ptr(hi), _ptr(lo), _ptr(out), _ptr(score) if score is not None else None,
        _ptr(changed) if changed is not None else None, ctypes.byref(ctr), int(threads),
    )
    if rc:
        raise OracleError(rc, "replay")
    digest = hashlib.sha256(out.astype("<u2", copy=False).tobytes(order="C")).hexdigest()
    res = OracleResult(
        output_rgb16=out,
        output_sha256=digest,
        attempted_pixels=ctr.attempted,
        written_pixels=ctr.written,
        public_rng_advances=ctr.public_advances,
        final_rng_state=ctr.final_state,
        changed_pixels=ctr.changed,
        startup_attempted=tuple(ctr.startup_attempted),
        startup_advances=tuple(ctr.startup_advances),
        startup_final_state=ctr.startup_final_state,
        stages=stages,
    )
    if diagnostics:
        floor = np.float32((params or Params()).score_floor)
        res.score_plane = score
        res.at_floor_mask = score == floor
        res.changed_mask = changed.astype(bool)
    return res


def process(main: np.ndarray, prepass: np.ndarray, *, threads: int = 0,
            diagnostics: bool = True) -> OracleResult:
    """engine.py:110-267 for the frozen LS-5000 profile."""

    payload, _, _ = prepass_reduce(prepass)
    alpha = np.frombuffer(payload, "<f4", 1, 0x04)[0]
    if float(1.0 - float(alpha)) == 0.0:  # profile.py:325-332
        raise ValueError("prepass alpha cannot equal one")
    rows = producer_rows(main)
    stages = stage_table(rows)
    res = replay(main, stages, threads=threads, diagnostics=diagnostics)
    res.prepass_payload = payload
    res.extra["producer"] = rows
    return res
