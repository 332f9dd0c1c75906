"""Batched processing: many frames of uneven sizes in flight on one B200.

No counterpart in the reference, which processes one job per call.  Each
frame is an independent job (its own prelude and its own RNG chain from the
job's initial state), so frames can run concurrently without changing any
result: up to ``slots`` frames are in flight, each in its own context slot
with its own CUDA stream and device buffers, and the kernels of different
frames overlap on the device (one frame's latency-bound walk and one-block
scans leave most SMs to the others).

* :func:`run_device_batch` -- frames already in device memory (pointers),
  outputs written to device memory; the measurement path.
* :func:`process_batch` -- :class:`ProcessingJob` objects in, reference-shaped
  :class:`ProcessingResult` objects out (host buffers), same validation and
  fail-closed behaviour as :func:`fauxice_b200.engine.process_b200`.
* :func:`tune_slots` -- picks the slot count, walk wave and stencil tile
  height that maximise throughput on a sample of the workload (the batching
  autotuner); :func:`autotune` caches that choice as JSON, keyed by device
  and frame shapes.  Every choice computes the same bits; only the time
  differs.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from .engine import (
    NIKON_PE_INITIAL_STATE,
    FrameOutcome,
    ProcessingResult,
    context,
    make_diagnostics,
    raise_library_error,
    reduce_prepass,
    replay_result,
)
from .profile import DEFAULT_PROFILE

FX_PENDING = 18


@dataclass
class DeviceFrame:
    """One device-resident frame: RGBI input and RGB16 output (device
    pointers as integers), optional score plane and changed mask."""

    rgbi: int
    height: int
    width: int
    rgb_out: int
    score_out: int = 0
    changed_out: int = 0
    rng_state: int = NIKON_PE_INITIAL_STATE


def _check(ctx: _lib.Context, status: int) -> None:
    if status:
        try:
            ctx.check(status)
        except _lib.LibraryError as error:
            raise_library_error(error)


def set_slots(ctx: _lib.Context, slots: int) -> None:
    with ctx.lock:
        _check(ctx, _lib.load().fx_set_slots(ctx.handle, int(slots)))


def reserve_frames(ctx: _lib.Context, max_height: int, max_width: int) -> None:
    """Size every slot for frames up to max_height x max_width now, so that no
    frame of the run reallocates device memory while others are in flight."""

    with ctx.lock:
        _check(ctx, _lib.load().fx_reserve_frames(ctx.handle, int(max_height), int(max_width)))


def set_walk_wave(ctx: _lib.Context, segments: int) -> None:
    """Segments per speculative walk wave (0: the default, three per SM)."""

    with ctx.lock:
        _check(ctx, _lib.load().fx_set_walk_wave(ctx.handle, int(segments)))


def set_stencil_tile(ctx: _lib.Context, rows: int) -> None:
    """Stencil tile height: 8 rows (four blocks per SM) or 16 (two)."""

    with ctx.lock:
        _check(ctx, _lib.load().fx_set_stencil_tile(ctx.handle, int(rows)))


def set_launch_priority(ctx: _lib.Context, enable: bool) -> None:
    """Launch the latency-bound kernels (producer scan, writer chain, walk)
    at the device's greatest priority (the default), or every kernel at the
    default priority."""

    with ctx.lock:
        _check(ctx, _lib.load().fx_set_launch_priority(ctx.handle, 1 if enable else 0))


def run_device_batch(ctx: _lib.Context, frames: Sequence[DeviceFrame], *, slots: int = 4,
                     params: _lib.FxParams | None = None) -> list[_lib.FxCounters]:
    """Process device-resident frames with up to ``slots`` in flight.

    Frames are submitted in order; when every slot is busy the oldest
    request is waited for.  Returns the counters of every frame, in order.
    """

    lib = _lib.load()
    set_slots(ctx, slots)
    if frames:
        reserve_frames(ctx, max(f.height for f in frames), max(f.width for f in frames))
    if params is None:
        params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    pending: deque[tuple[int, int]] = deque()  # (frame index, ticket)
    results: list[_lib.FxCounters | None] = [None] * len(frames)

    def wait_oldest() -> None:
        index, ticket = pending.popleft()
        counters = _lib.FxCounters()
        status = lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters))
        _check(ctx, status)
        results[index] = counters

    for index, f in enumerate(frames):
        if len(pending) >= slots:  # the context may hold more slots than asked for
            wait_oldest()
        while True:
            ticket = ctypes.c_int64()
            with ctx.lock:
                status = lib.fx_submit_device(
                    ctx.handle, ctypes.c_void_p(f.rgbi), f.height, f.width, ctypes.byref(params),
                    None, int(f.rng_state) & 0xFFFFFF, ctypes.c_void_p(f.rgb_out),
                    ctypes.c_void_p(f.score_out or None), ctypes.c_void_p(f.changed_out or None),
                    ctypes.byref(ticket))
            if status == FX_PENDING and pending:
                wait_oldest()
                continue
            _check(ctx, status)
            pending.append((index, ticket.value))
            break
    while pending:
        wait_oldest()
    return results  # type: ignore[return-value]


def tune_slots(ctx: _lib.Context, frames: Sequence[DeviceFrame],
               candidates: Iterable[int] = (1, 2, 4, 8), waves: Iterable[int] = (0,),
               repeats: int = 1, tiles: Iterable[int] = (8,)) -> tuple[tuple[int, ...], dict]:
    """Time the sample batch at each (slots, walk wave, stencil tile)
    combination; leave the best walk wave and tile set and return the
    choice with the measured seconds of every combination (after one
    warm-up run that allocates the slots' buffers).  The choice is a
    (slots, wave) pair when only one tile height is tried, else
    (slots, wave, tile)."""

    candidates, waves, tiles = tuple(candidates), tuple(waves), tuple(tiles)
    timings: dict[tuple[int, ...], float] = {}
    run_device_batch(ctx, frames, slots=max(candidates))
    import torch

    for tile in tiles:
        set_stencil_tile(ctx, tile)
        for wave in waves:
            set_walk_wave(ctx, wave)
            for slots in candidates:
                best = float("inf")
                for _ in range(repeats):
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    run_device_batch(ctx, frames, slots=slots)
                    torch.cuda.synchronize()
                    best = min(best, time.perf_counter() - t0)
                key = (slots, wave) if len(tiles) == 1 else (slots, wave, tile)
                timings[key] = best
    choice = min(timings, key=timings.get)
    set_walk_wave(ctx, choice[1])
    set_stencil_tile(ctx, choice[2] if len(choice) > 2 else tiles[0])
    return choice, timings


def tuning_cache_path() -> str:
    """Where autotune keeps its choices: FAUXICE_B200_TUNING, else
    $XDG_CACHE_HOME (or ~/.cache)/fauxice_b200/tuning.json."""

    path = os.environ.get("FAUXICE_B200_TUNING")
    if path:
        return path
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "fauxice_b200", "tuning.json")


def tuning_key(device: int, frames: Sequence[DeviceFrame]) -> str:
    """Device name, SM count and the sorted set of frame shapes."""

    import torch

    props = torch.cuda.get_device_properties(device)
    shapes = sorted({(f.height, f.width) for f in frames})
    return (f"{props.name}|sm{props.major}{props.minor}|{props.multi_processor_count}SM|"
            + ",".join(f"{h}x{w}" for h, w in shapes))


def autotune(ctx: _lib.Context, frames: Sequence[DeviceFrame], *,
             candidates: Iterable[int] = (2, 4, 8), waves: Iterable[int] = (0, 148),
             tiles: Iterable[int] = (8, 16), cache_path: str | None = None,
             retune: bool = False) -> tuple[dict, bool]:
    """The batching configuration for this device and these frame shapes:
    from the JSON cache when an entry exists (and ``retune`` is off), else
    measured with :func:`tune_slots` over every combination and stored.
    Applies the walk wave and stencil tile to the context and returns
    ({"slots", "walk_wave", "stencil_tile", "timings_ms"}, from_cache)."""

    path = cache_path or tuning_cache_path()
    key = tuning_key(ctx.device, frames)
    cache: dict = {}
    try:
        with open(path) as handle:
            cache = json.load(handle)
    except (OSError, ValueError):
        cache = {}
    entry = None if retune else cache.get(key)
    from_cache = entry is not None
    if entry is None:
        choice, timings = tune_slots(ctx, frames, candidates=candidates, waves=waves,
                                     tiles=tuple(tiles))
        if len(choice) == 2:
            choice = (*choice, tuple(tiles)[0])
        entry = {"slots": choice[0], "walk_wave": choice[1], "stencil_tile": choice[2],
                 "timings_ms": {",".join(str(v) for v in k): round(1e3 * t, 2)
                                for k, t in timings.items()}}
        cache[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as handle:
            json.dump(cache, handle, indent=1, sort_keys=True)
        os.replace(tmp, path)
    set_walk_wave(ctx, entry["walk_wave"])
    set_stencil_tile(ctx, entry["stencil_tile"])
    return entry, from_cache


def _sha256(array: np.ndarray) -> bytes:
    # little-endian uint16 bytes in row-major order, hashed in place (hashlib
    # releases the GIL for large buffers, so several frames hash at once)
    return hashlib.sha256(memoryview(array).cast("B")).digest()


def process_batch(jobs: Sequence, *, slots: int = 4, export_diagnostics: bool = False,
                  device: int = 0, hash_workers: int | None = None) -> list[ProcessingResult]:
    """Process many jobs with up to ``slots`` frames in flight.

    Every job is validated (and its prepass record checked) before any is
    submitted, so a bad job fails the call before device work starts.  Each
    result equals :func:`fauxice_b200.engine.process_b200` on the same job.
    The output digests (the replay result's output_sha256) are computed on
    ``hash_workers`` threads while later frames are still on the device.
    """

    for job in jobs:
        DEFAULT_PROFILE.validate_job(job)
    ctx = context(device)
    for job in jobs:
        payload, _, _ = reduce_prepass(ctx, job.acquisition.prepass.pixels)
        DEFAULT_PROFILE.check_prepass_record(payload)
    lib = _lib.load()
    set_slots(ctx, slots)
    if jobs:
        shapes = [job.acquisition.main.pixels.shape for job in jobs]
        reserve_frames(ctx, max(int(sh[0]) for sh in shapes), max(int(sh[1]) for sh in shapes))
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    floor = DEFAULT_PROFILE.score_floor()

    inflight: deque[tuple[int, int, object]] = deque()
    finished: list[tuple[int, FrameOutcome, object]] = []
    hasher = ThreadPoolExecutor(hash_workers or min(8, os.cpu_count() or 1))

    def finish_oldest() -> None:
        index, ticket, keep = inflight.popleft()
        counters = _lib.FxCounters()
        status = lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters))
        _check(ctx, status)
        _, out, score, changed = keep
        finished.append((index, FrameOutcome(out, counters, score, changed),
                         hasher.submit(_sha256, out)))

    for index, job in enumerate(jobs):
        px = np.ascontiguousarray(job.acquisition.main.pixels, dtype=np.uint16)
        h, w = px.shape[:2]
        out = np.empty((h, w, 3), np.uint16)
        score = np.empty((h, w), np.float32) if export_diagnostics else None
        changed = np.empty((h, w), np.uint8) if export_diagnostics else None
        frame = _lib.FxFrame(
            main_rgbi=px.ctypes.data, height=h, width=w, params=ctypes.pointer(params),
            stages=None, rng_state=NIKON_PE_INITIAL_STATE, rgb_out=out.ctypes.data,
            score_out=score.ctypes.data if score is not None else None,
            changed_out=changed.ctypes.data if changed is not None else None)
        if len(inflight) >= slots:
            finish_oldest()
        while True:
            ticket = ctypes.c_int64()
            with ctx.lock:
                status = lib.fx_submit(ctx.handle, ctypes.byref(frame), ctypes.byref(ticket))
            if status == FX_PENDING and inflight:
                finish_oldest()
                continue
            _check(ctx, status)
            inflight.append((index, ticket.value, (px, out, score, changed)))
            break
    try:
        while inflight:
            finish_oldest()
        results: list[ProcessingResult | None] = [None] * len(jobs)
        for index, outcome, digest in finished:
            outcome.digest = digest.result()
            diagnostics = make_diagnostics(outcome, floor) if export_diagnostics else None
            results[index] = ProcessingResult(output_rgb16=outcome.output,
                                              replay=replay_result(outcome),
                                              profile_id=DEFAULT_PROFILE.profile_id,
                                              diagnostics=diagnostics)
    finally:
        hasher.shutdown(wait=True)
    return results  # type: ignore[return-value]
