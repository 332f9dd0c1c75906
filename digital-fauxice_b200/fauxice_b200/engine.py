"""B200 execution of one supported job, behind the reference's backend contract.

``process_b200`` has the signature of the reference's ``process_cuda``
(cuda_backend/process.py:25-33) and follows the shared orchestration of
``_run_supported_job`` (engine.py:110-267): validate first, fail closed
before any work when the backend cannot run, report the VALIDATING ->
PREPASS -> PRODUCER -> RECONSTRUCTION -> COMPLETE phases, honour
cooperative cancellation between phases, and write a caller-owned output
only after full success.  The main-pass work (producer schedule, stage
table, planes, stencil, hidden startup replay, dither writer, emit,
counters, diagnostics) runs on the GPU through libfauxice_b200.
"""

from __future__ import annotations

import hashlib
import threading
import time
from collections.abc import Callable
from dataclasses import dataclass
from enum import Enum

import numpy as np
import numpy.typing as npt

from . import _lib
from .profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE, factor_tables, response_lut


class ProcessingPhase(str, Enum):
    VALIDATING = "validating"
    PREPASS = "prepass"
    PRODUCER = "producer"
    RECONSTRUCTION = "reconstruction"
    COMPLETE = "complete"


@dataclass(frozen=True)
class ProcessingProgress:
    phase: ProcessingPhase
    completed: int
    total: int
    attempted_pixels: int = 0
    written_pixels: int = 0


@dataclass(frozen=True)
class ProcessingDiagnostics:
    """engine.py:39-66: score plane, its floor, at-floor and changed masks."""

    score_plane: npt.NDArray[np.float32]
    score_floor: np.float32
    at_floor_mask: npt.NDArray[np.bool_]
    changed_mask: npt.NDArray[np.bool_]

    def __post_init__(self) -> None:
        if self.score_plane.dtype != np.dtype(np.float32):
            raise ValueError("diagnostic score plane must be float32")
        if self.score_plane.ndim != 2:
            raise ValueError("diagnostic score plane must be HxW")
        floor = np.asarray(self.score_floor)
        if floor.dtype != np.dtype(np.float32) or floor.ndim != 0:
            raise ValueError("diagnostic score floor must be a float32 scalar")
        if not np.isfinite(floor) or floor <= np.float32(0.0):
            raise ValueError("diagnostic score floor must be finite and positive")
        for name, mask in (("at-floor", self.at_floor_mask), ("changed", self.changed_mask)):
            if mask.dtype != np.dtype(np.bool_):
                raise ValueError(f"diagnostic {name} mask must be bool")
            if mask.shape != self.score_plane.shape:
                raise ValueError(f"diagnostic {name} mask must have shape "
                                 f"{self.score_plane.shape}")


@dataclass(frozen=True)
class StartupReplayResult:
    """startup.py:37-43."""

    attempted_per_stage: tuple[int, int, int, int, int, int]
    rng_advances_per_stage: tuple[int, int, int, int, int, int]
    final_rng_state: int


@dataclass(frozen=True)
class StreamingReplayResult:
    """streaming.py:63-75."""

    shape: tuple[int, int, int]
    startup: StartupReplayResult | None
    attempted_pixels: int
    written_pixels: int
    public_rng_advances: int
    final_rng_state: int
    output_sha256: str
    changed_pixels: int


@dataclass(frozen=True)
class ProcessingResult:
    """engine.py:69-74."""

    output_rgb16: npt.NDArray[np.uint16]
    replay: StreamingReplayResult
    profile_id: str
    diagnostics: ProcessingDiagnostics | None = None


class ProcessingCancelled(RuntimeError):
    """Raised when a caller requests cooperative cancellation."""


class B200BackendUnavailable(RuntimeError):
    """The B200 backend was requested but cannot run exactly here."""


ProgressCallback = Callable[[ProcessingProgress], None]
CancellationCallback = Callable[[], bool]

_STATUS_ERRORS = {
    5: ValueError,   # non-finite auxiliary
    6: ValueError,   # non-finite work value
    7: ValueError,   # combiner inputs
    8: ValueError,   # dither inputs
    9: ValueError,   # setter scale == 1
    10: ValueError,  # non-finite stage calibration
    12: ValueError,  # geometry
}

_CONTEXTS: dict[int, _lib.Context] = {}
_CONTEXT_LOCK = threading.Lock()


def context(device: int = 0) -> _lib.Context:
    """The per-process device context, created on first use (fail closed)."""

    with _CONTEXT_LOCK:
        ctx = _CONTEXTS.get(device)
        if ctx is not None:
            return ctx
        try:
            _lib.load()
        except Exception as error:
            raise B200BackendUnavailable(f"libfauxice_b200 is not loadable: {error}") from error
        status, reason = _lib.device_check(device)
        if status:
            raise B200BackendUnavailable(reason)
        try:
            lut = response_lut()
            high, low = factor_tables()
        except Exception as error:
            raise B200BackendUnavailable(str(error)) from error
        try:
            ctx = _lib.Context(device, lut=lut, high=high, low=low)
        except _lib.LibraryError as error:
            raise B200BackendUnavailable(str(error)) from error
        # fx_process hashes the output while it is still being copied back
        ctx.check(_lib.load().fx_set_output_digest(ctx.handle, 1))
        _CONTEXTS[device] = ctx
        return ctx


def raise_library_error(error: _lib.LibraryError) -> None:
    cls = _STATUS_ERRORS.get(error.status)
    if cls is not None:
        raise cls(str(error)) from error
    if error.status == 11:
        from .profile import UnboundBehaviorError

        raise UnboundBehaviorError(str(error)) from error
    raise B200BackendUnavailable(str(error)) from error


def _notify(callback, phase, completed, total, attempted=0, written=0) -> None:
    if callback is not None:
        callback(ProcessingProgress(phase, completed, total, attempted, written))


def _check_cancelled(cancelled: CancellationCallback | None) -> None:
    if cancelled is not None and cancelled():
        raise ProcessingCancelled("portable correction was cancelled")


def reduce_prepass(ctx: _lib.Context, prepass: np.ndarray) -> tuple[bytes, int, int]:
    """prepass.py:96-236 through fx_reduce_prepass."""

    import ctypes

    px = np.ascontiguousarray(prepass, dtype=np.uint16)
    payload = (ctypes.c_uint8 * 64)()
    valid = ctypes.c_int64()
    tiles = ctypes.c_int64()
    lut = ctx._tables[0]
    status = _lib.load().fx_reduce_prepass(_lib.ptr(px), px.shape[0], px.shape[1], _lib.ptr(lut),
                                           payload, ctypes.byref(valid), ctypes.byref(tiles))
    if status:
        raise ValueError(f"prepass reduction failed (status {status})")
    return bytes(payload), valid.value, tiles.value


@dataclass
class FrameOutcome:
    output: np.ndarray
    counters: _lib.FxCounters
    score: np.ndarray | None
    changed: np.ndarray | None
    digest: bytes | None = None  # SHA-256 of the output, when the library computed it


def run_frame(ctx: _lib.Context, main: np.ndarray, params: _lib.FxParams,
              stages: np.ndarray | None, rng_state: int, diagnostics: bool) -> FrameOutcome:
    """One synchronous fx_process call."""

    import ctypes

    px = np.ascontiguousarray(main, dtype=np.uint16)
    h, w = px.shape[:2]
    out = np.empty((h, w, 3), np.uint16)
    score = np.empty((h, w), np.float32) if diagnostics else None
    changed = np.empty((h, w), np.uint8) if diagnostics else None
    if stages is not None:
        stages = np.ascontiguousarray(stages, dtype=_lib.STAGE_DTYPE)
        if stages.shape != (h + 6,):
            raise ValueError("stage table must hold height + 6 entries")
    frame = _lib.FxFrame(
        main_rgbi=px.ctypes.data, height=h, width=w, params=ctypes.pointer(params),
        stages=stages.ctypes.data if stages is not None else None,
        rng_state=int(rng_state) & 0xFFFFFF, rgb_out=out.ctypes.data,
        score_out=score.ctypes.data if score is not None else None,
        changed_out=changed.ctypes.data if changed is not None else None,
    )
    counters = _lib.FxCounters()
    digest = None
    with ctx.lock:
        lib = _lib.load()
        status = lib.fx_process(ctx.handle, ctypes.byref(frame), ctypes.byref(counters))
        if status:
            try:
                ctx.check(status)
            except _lib.LibraryError as error:
                raise_library_error(error)
        buf = (ctypes.c_uint8 * 32)()
        if lib.fx_output_digest(ctx.handle, buf) == 0:
            digest = bytes(buf)
    return FrameOutcome(out, counters, score, changed, digest)


_CANCEL_POLL_S = 0.0005  # how often a running pass checks the cancellation callback


def run_frame_cancellable(ctx: _lib.Context, main: np.ndarray, params: _lib.FxParams,
                          stages: np.ndarray | None, rng_state: int, diagnostics: bool,
                          cancelled: CancellationCallback) -> FrameOutcome:
    """One frame through fx_submit / fx_fetch, polling ``cancelled`` while
    the device works.

    The reference polls its callback between phases (engine.py:103-106); here
    the pass itself is the long phase, so the callback is polled while it
    runs and a True answer is handed to the device with fx_cancel: the pass
    stops at its next stage boundary, and nothing is copied to the caller.
    """

    import ctypes

    px = np.ascontiguousarray(main, dtype=np.uint16)
    h, w = px.shape[:2]
    if stages is not None:
        stages = np.ascontiguousarray(stages, dtype=_lib.STAGE_DTYPE)
        if stages.shape != (h + 6,):
            raise ValueError("stage table must hold height + 6 entries")
    # rgb_out NULL: the results stay staged in the library until fx_fetch
    frame = _lib.FxFrame(
        main_rgbi=px.ctypes.data, height=h, width=w, params=ctypes.pointer(params),
        stages=stages.ctypes.data if stages is not None else None,
        rng_state=int(rng_state) & 0xFFFFFF, rgb_out=None, score_out=None, changed_out=None)
    lib = _lib.load()

    def check(status: int) -> None:
        if status:
            try:
                ctx.check(status)
            except _lib.LibraryError as error:
                raise_library_error(error)

    with ctx.lock:
        ticket = ctypes.c_int64()
        check(lib.fx_submit(ctx.handle, ctypes.byref(frame), ctypes.byref(ticket)))
        while True:
            status = lib.fx_poll(ctx.handle, ticket.value)
            if status != _lib.FX_PENDING:
                break
            if cancelled():
                lib.fx_cancel(ctx.handle, ticket.value)
                # releases the slot; the staged results are dropped
                lib.fx_fetch(ctx.handle, ticket.value, -1, None, None, None, None, None)
                raise ProcessingCancelled("portable correction was cancelled")
            time.sleep(_CANCEL_POLL_S)
        out = np.empty((h, w, 3), np.uint16)
        score = np.empty((h, w), np.float32) if diagnostics else None
        changed = np.empty((h, w), np.uint8) if diagnostics else None
        counters = _lib.FxCounters()
        check(lib.fx_fetch(ctx.handle, ticket.value, -1, _lib.ptr(out), ctypes.byref(counters),
                           _lib.ptr(score), None, _lib.ptr(changed)))
    return FrameOutcome(out, counters, score, changed)


def replay_result(outcome: FrameOutcome) -> StreamingReplayResult:
    c = outcome.counters
    h, w = outcome.output.shape[:2]
    if outcome.digest is not None:  # hashed by the library during the download
        hexdigest = outcome.digest.hex()
    else:
        # little-endian uint16 bytes in row-major order, hashed in place (no copy)
        out = np.ascontiguousarray(outcome.output.astype("<u2", copy=False))
        hexdigest = hashlib.sha256(memoryview(out).cast("B")).hexdigest()
    return StreamingReplayResult(
        shape=(h, w, 3),
        startup=StartupReplayResult(
            attempted_per_stage=tuple(int(v) for v in c.startup_attempted),
            rng_advances_per_stage=tuple(int(v) for v in c.startup_advances),
            final_rng_state=int(c.startup_final_state),
        ),
        attempted_pixels=int(c.attempted),
        written_pixels=int(c.written),
        public_rng_advances=int(c.public_advances),
        final_rng_state=int(c.final_state),
        output_sha256=hexdigest,
        changed_pixels=int(c.changed),
    )


def make_diagnostics(outcome: FrameOutcome, floor: np.float32) -> ProcessingDiagnostics:
    score = outcome.score
    at_floor = np.ascontiguousarray(score == floor)
    changed = np.ascontiguousarray(outcome.changed.astype(bool))
    for array in (score, at_floor, changed):
        array.setflags(write=False)
    return ProcessingDiagnostics(score_plane=score, score_floor=np.float32(floor),
                                 at_floor_mask=at_floor, changed_mask=changed)


def process_b200(
    job,
    *,
    output_rgb16: npt.NDArray[np.uint16] | None = None,
    progress: ProgressCallback | None = None,
    cancelled: CancellationCallback | None = None,
    stage_timings: dict | None = None,
    export_diagnostics: bool = False,
    device: int = 0,
) -> ProcessingResult:
    """Process one validated LS-5000 selector-8 Normal acquisition on a B200.

    A caller-owned output is committed only after successful completion;
    validation errors, backend refusal and cancellation leave it unchanged.
    """

    timer = time.perf_counter
    t0 = timer()
    _notify(progress, ProcessingPhase.VALIDATING, 0, 1)
    DEFAULT_PROFILE.validate_job(job)
    ctx = context(device)  # fail closed before any work
    main_pixels = job.acquisition.main.pixels
    expected_shape = (*main_pixels.shape[:2], 3)
    destination = None
    if output_rgb16 is not None:
        destination = np.asarray(output_rgb16)
        if destination.dtype != np.dtype(np.uint16) or destination.shape != expected_shape:
            raise ValueError(f"output must be writable uint16 with shape {expected_shape}")
        if not destination.flags.writeable:
            raise ValueError("output must be writable")
    _check_cancelled(cancelled)
    _notify(progress, ProcessingPhase.VALIDATING, 1, 1)

    t1 = timer()
    _notify(progress, ProcessingPhase.PREPASS, 0, 1)
    payload, _, _ = reduce_prepass(ctx, job.acquisition.prepass.pixels)
    DEFAULT_PROFILE.check_prepass_record(payload)
    _check_cancelled(cancelled)
    _notify(progress, ProcessingPhase.PREPASS, 1, 1)

    # The producer schedule and stage table are derived on the device as the
    # first kernels of the main pass (fx_process with no host stage table).
    _notify(progress, ProcessingPhase.PRODUCER, 0, 1)
    _check_cancelled(cancelled)
    _notify(progress, ProcessingPhase.PRODUCER, 1, 1)

    t2 = timer()
    height = int(main_pixels.shape[0])
    _notify(progress, ProcessingPhase.RECONSTRUCTION, 0, height)
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    if cancelled is None:
        outcome = run_frame(ctx, main_pixels, params, None, NIKON_PE_INITIAL_STATE,
                            export_diagnostics)
    else:
        outcome = run_frame_cancellable(ctx, main_pixels, params, None, NIKON_PE_INITIAL_STATE,
                                        export_diagnostics, cancelled)
    replay = replay_result(outcome)
    _notify(progress, ProcessingPhase.RECONSTRUCTION, height, height, replay.attempted_pixels,
            replay.written_pixels)
    _check_cancelled(cancelled)
    t3 = timer()

    diagnostics = None
    if export_diagnostics:
        diagnostics = make_diagnostics(outcome, DEFAULT_PROFILE.score_floor())
    if destination is None:
        output = outcome.output
    else:
        np.copyto(destination, outcome.output)
        output = destination
    _notify(progress, ProcessingPhase.COMPLETE, 1, 1)
    if stage_timings is not None:
        stage_timings.update({"validate_s": t1 - t0, "prepass_s": t2 - t1,
                              "device_pass_s": t3 - t2, "total_s": timer() - t0})
    return ProcessingResult(output_rgb16=output, replay=replay, profile_id=DEFAULT_PROFILE.profile_id,
                            diagnostics=diagnostics)
