"""ctypes binding of libfauxice_b200.so (the C ABI in include/fauxice_b200.h).

There is no CPU fallback: if the library or a usable sm_100 device is
missing, every entry point raises instead of computing anything.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfauxice_b200.so")

FX_OK = 0
FX_PENDING = 18
STATUS_NAMES = {
    1: "invalid argument",
    2: "no CUDA device",
    3: "unsupported device",
    4: "out of device memory",
    5: "non-finite auxiliary",
    6: "non-finite work value",
    7: "non-finite combiner input",
    8: "non-finite dither input",
    9: "setter scale equals one",
    10: "non-finite stage calibration",
    11: "alpha==1 without replacement",
    12: "unsupported geometry",
    13: "cancelled",
    14: "timeout",
    15: "CUDA runtime error",
    16: "internal consistency check failed",
    17: "tables not set",
    18: "pending",
}


class LibraryError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, status: int, message: str) -> None:
        super().__init__(message)
        self.status = status


class FxParams(ctypes.Structure):
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


class FxCounters(ctypes.Structure):
    _fields_ = [
        ("attempted", ctypes.c_int64),
        ("written", ctypes.c_int64),
        ("public_advances", ctypes.c_int64),
        ("changed", ctypes.c_int64),
        ("final_state", ctypes.c_uint32),
        ("startup_final_state", ctypes.c_uint32),
        ("startup_attempted", ctypes.c_int64 * 6),
        ("startup_advances", ctypes.c_int64 * 6),
        ("rng_dependent", ctypes.c_int64),
        ("walk_fallbacks", ctypes.c_int64),
        ("walk_candidate_steps", ctypes.c_int64),
        ("walk_candidates", ctypes.c_int64),
        ("walk_survivors", ctypes.c_int64),
        ("walk_packed_segments", ctypes.c_int64),
        ("capacity_reruns", ctypes.c_int64),
    ]


class FxFrame(ctypes.Structure):
    _fields_ = [
        ("main_rgbi", ctypes.c_void_p),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("params", ctypes.POINTER(FxParams)),
        ("stages", ctypes.c_void_p),
        ("rng_state", ctypes.c_uint32),
        ("rgb_out", ctypes.c_void_p),
        ("score_out", ctypes.c_void_p),
        ("changed_out", ctypes.c_void_p),
    ]


# Every exported symbol of include/fauxice_b200.h with its ctypes signature.
_P = ctypes.c_void_p
SIGNATURES = {
    "fx_version": ([], ctypes.c_int),
    "fx_device_check": ([ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "fx_context_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "fx_context_destroy": ([_P], None),
    "fx_last_error": ([_P, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "fx_set_tables": ([_P, _P, _P, _P], ctypes.c_int),
    "fx_reduce_prepass": ([_P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P], ctypes.c_int),
    "fx_producer_rows": ([_P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P], ctypes.c_int),
    "fx_producer_rows_static": ([_P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
                                ctypes.c_int),
    "fx_stage_table": ([ctypes.c_int32, _P, _P, _P, _P, ctypes.c_float, _P], ctypes.c_int),
    "fx_process": ([_P, ctypes.POINTER(FxFrame), ctypes.POINTER(FxCounters)], ctypes.c_int),
    "fx_process_device": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(FxParams), _P,
                           ctypes.c_uint32, _P, _P, _P, _P, ctypes.POINTER(FxCounters)],
                          ctypes.c_int),
    "fx_sync_counters": ([_P, ctypes.POINTER(FxCounters)], ctypes.c_int),
    "fx_set_slots": ([_P, ctypes.c_int32], ctypes.c_int),
    "fx_set_parallel_walk": ([_P, ctypes.c_int], ctypes.c_int),
    "fx_set_walk_wave": ([_P, ctypes.c_int32], ctypes.c_int),
    "fx_set_launch_priority": ([_P, ctypes.c_int], ctypes.c_int),
    "fx_set_output_digest": ([_P, ctypes.c_int], ctypes.c_int),
    "fx_reserve_frames": ([_P, ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "fx_output_digest": ([_P, _P], ctypes.c_int),
    "fx_submit": ([_P, ctypes.POINTER(FxFrame), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "fx_submit_device": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(FxParams), _P,
                          ctypes.c_uint32, _P, _P, _P, ctypes.POINTER(ctypes.c_int64)],
                         ctypes.c_int),
    "fx_poll": ([_P, ctypes.c_int64], ctypes.c_int),
    "fx_wait": ([_P, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(FxCounters)], ctypes.c_int),
    "fx_cancel": ([_P, ctypes.c_int64], ctypes.c_int),
    "fx_release_idle_slots": ([_P, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "fx_reserve_slots": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "fx_fetch": ([_P, ctypes.c_int64, ctypes.c_int64, _P, ctypes.POINTER(FxCounters), _P, _P, _P],
                 ctypes.c_int),
    "fx_set_walk_window": ([_P, ctypes.c_double], ctypes.c_int),
    "fx_set_stencil_tile": ([_P, ctypes.c_int32], ctypes.c_int),
    "fx_set_list_capacity": ([_P, ctypes.c_int64], ctypes.c_int),
    "fx_mem_info": ([_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)],
                    ctypes.c_int),
    "fx_frame_bytes": ([ctypes.c_int32, ctypes.c_int32], ctypes.c_int64),
    "fx_pass_bytes": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)],
                      ctypes.c_int),
    "fx_profile_enable": ([_P, ctypes.c_int], ctypes.c_int),
    "fx_profile_read": ([_P, _P, ctypes.POINTER(ctypes.c_int64), ctypes.c_int], ctypes.c_int),
    # at-floor routing census primitives
    "fx_label8": ([_P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P,
                   ctypes.POINTER(ctypes.c_int64), _P], ctypes.c_int),
    "fx_chessboard_distance": ([_P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P],
                               ctypes.c_int),
    "fx_label_stats": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, _P, _P, _P, _P],
                       ctypes.c_int),
    "fx_dilate_square": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
                         ctypes.c_int),
    "fx_label_pairs": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, _P, _P,
                        ctypes.POINTER(ctypes.c_int64), _P], ctypes.c_int),
    "fx_map_labels": ([_P, ctypes.c_int64, _P, ctypes.c_int64, _P, _P, _P], ctypes.c_int),
    "fx_clear_label": ([_P, _P, ctypes.c_int64, ctypes.c_int32, _P,
                        ctypes.POINTER(ctypes.c_int64), _P], ctypes.c_int),
    "fx_count_where": ([_P, _P, ctypes.c_int64, ctypes.c_int64, _P, _P], ctypes.c_int),
    "fx_tile_extract": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P], ctypes.c_int),
    "fx_census_provisional_json": ([ctypes.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                    ctypes.c_int64], ctypes.c_int64),
    "fx_census_final_json": ([ctypes.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int64],
                             ctypes.c_int64),
    "fx_tile_scatter": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P], ctypes.c_int),
}

PROFILE_STAGES = ("producer", "planes", "stencil", "startup", "chain", "walk", "apply")

_LIB = None
_LIB_LOCK = threading.Lock()


def load() -> ctypes.CDLL:
    """Load the library (raises OSError / RuntimeError when it is unusable)."""

    global _LIB
    with _LIB_LOCK:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"{LIB_PATH} is missing; run digital-fauxice_b200/build.py")
            handle = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.argtypes = args
                fn.restype = res
            if handle.fx_version() != 1:
                raise RuntimeError("libfauxice_b200 ABI version mismatch")
            _LIB = handle
        return _LIB


def ptr(array: np.ndarray | None) -> ctypes.c_void_p | None:
    if array is None:
        return None
    return ctypes.c_void_p(array.ctypes.data)


def device_check(device: int = 0) -> tuple[int, str]:
    buf = ctypes.create_string_buffer(256)
    status = load().fx_device_check(device, buf, len(buf))
    return status, buf.value.decode()


class Context:
    """One device context: tables uploaded once, frame buffers reused."""

    def __init__(self, device: int = 0, *, lut=None, high=None, low=None) -> None:
        lib = load()
        handle = ctypes.c_void_p()
        status = lib.fx_context_create(device, ctypes.byref(handle))
        if status:
            raise LibraryError(status, self._error(None))
        self._lib = lib
        self.handle = handle
        self.device = device
        self.lock = threading.Lock()
        if lut is not None:
            self.set_tables(lut, high, low)

    def _error(self, handle) -> str:
        buf = ctypes.create_string_buffer(512)
        load().fx_last_error(handle, buf, len(buf))
        return buf.value.decode()

    def check(self, status: int) -> None:
        if status:
            raise LibraryError(status, self._error(self.handle) or STATUS_NAMES.get(status, ""))

    def set_tables(self, lut: np.ndarray, high: np.ndarray, low: np.ndarray) -> None:
        self._tables = (np.ascontiguousarray(lut, np.float32), np.ascontiguousarray(high, np.uint32),
                        np.ascontiguousarray(low, np.uint32))
        self.check(self._lib.fx_set_tables(self.handle, *(ptr(t) for t in self._tables)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.fx_context_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown
        try:
            self.close()
        except Exception:
            pass
