"""Serving: requests of mixed sizes admitted as they arrive (continuous batching).

No counterpart in the reference.  A request is one RGBI frame in host
memory.  The loop admits requests in arrival order while a context slot is
free and the device has room for the frame's working set (free HBM from
fx_mem_info against fx_frame_bytes plus the request's own input/output
buffers), so frames that arrive while others run are processed alongside
them.  Each admitted frame is copied to the device, submitted with
fx_submit_device, and polled; its latency runs from arrival to the moment
its completion is seen.  Results equal one-frame processing: every request
is an independent job.

Device memory for inputs and outputs is plumbing (torch tensors); the
processing itself is the library's.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib, batch
from .engine import NIKON_PE_INITIAL_STATE
from .profile import DEFAULT_PROFILE


@dataclass
class Request:
    arrival_s: float  # seconds after the start of the run
    pixels: object    # H x W x 4 uint16 in host memory: a numpy array, or a
                      # pinned torch int16 tensor (then the upload is a DMA)


@dataclass
class Completion:
    index: int
    arrival_s: float
    admitted_s: float
    done_s: float
    counters: _lib.FxCounters
    output: np.ndarray | None = None

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


@dataclass
class ServeReport:
    completions: list[Completion] = field(default_factory=list)
    wall_s: float = 0.0
    megapixels: float = 0.0

    def percentile_ms(self, q: float) -> float:
        lat = np.array([c.latency_s for c in self.completions]) * 1e3
        return float(np.percentile(lat, q)) if lat.size else float("nan")

    def summary(self) -> dict:
        return {"requests": len(self.completions), "wall_s": round(self.wall_s, 3),
                "mp_per_s": round(self.megapixels / self.wall_s, 1) if self.wall_s else None,
                "p50_ms": round(self.percentile_ms(50), 2),
                "p95_ms": round(self.percentile_ms(95), 2),
                "p99_ms": round(self.percentile_ms(99), 2)}


def poisson_arrivals(rate_per_s: float, duration_s: float, seed: int) -> np.ndarray:
    """Arrival times of a seeded Poisson process on [0, duration)."""

    rng = np.random.default_rng(seed)
    times, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate_per_s)
        if t >= duration_s:
            return np.array(times)
        times.append(t)


def serve(ctx: _lib.Context, requests: Sequence[Request], *, slots: int = 4,
          reserve_bytes: int = 2 << 30, keep_outputs: bool = False) -> ServeReport:
    """Run the request loop in real time; requests must be sorted by arrival."""

    import torch

    lib = _lib.load()
    batch.set_slots(ctx, slots)
    if requests:  # size the slots once: no reallocation while frames are in flight
        batch.reserve_frames(ctx, max(int(r.pixels.shape[0]) for r in requests),
                             max(int(r.pixels.shape[1]) for r in requests))
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    copy_stream = torch.cuda.Stream()
    report = ServeReport()
    waiting: deque[int] = deque()
    inflight: dict[int, tuple] = {}  # ticket -> (index, admitted, tensors)
    nxt = 0
    start = time.perf_counter()

    def now() -> float:
        return time.perf_counter() - start

    def room_for(h: int, w: int) -> bool:
        free, total = ctypes.c_size_t(), ctypes.c_size_t()
        with ctx.lock:
            if lib.fx_mem_info(ctx.handle, ctypes.byref(free), ctypes.byref(total)):
                return True
        need = lib.fx_frame_bytes(h, w) + (h * w * 14)
        return free.value >= need + reserve_bytes or len(inflight) == 0

    while nxt < len(requests) or waiting or inflight:
        t = now()
        while nxt < len(requests) and requests[nxt].arrival_s <= t:
            waiting.append(nxt)
            nxt += 1
        # admission: slot free and memory for the frame
        while waiting and len(inflight) < slots:
            i = waiting[0]
            src = requests[i].pixels
            h, w = int(src.shape[0]), int(src.shape[1])
            if not room_for(h, w):
                break
            waiting.popleft()
            if isinstance(src, np.ndarray):
                src = torch.from_numpy(np.ascontiguousarray(src, dtype=np.uint16).view(np.int16))
            with torch.cuda.stream(copy_stream):
                d_in = src.to("cuda", non_blocking=True)
                d_out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
            copy_stream.synchronize()
            ticket = ctypes.c_int64()
            with ctx.lock:
                status = lib.fx_submit_device(
                    ctx.handle, ctypes.c_void_p(d_in.data_ptr()), h, w, ctypes.byref(params),
                    None, NIKON_PE_INITIAL_STATE, ctypes.c_void_p(d_out.data_ptr()), None, None,
                    ctypes.byref(ticket))
            batch._check(ctx, status)
            inflight[ticket.value] = (i, now(), d_in, d_out)
        # completions
        finished = []
        for ticket in list(inflight):
            with ctx.lock:
                status = lib.fx_poll(ctx.handle, ticket)
            if status == batch.FX_PENDING:
                continue
            counters = _lib.FxCounters()
            status = lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters))
            batch._check(ctx, status)
            done = now()
            i, admitted, _, d_out = inflight.pop(ticket)
            output = d_out.cpu().numpy().view(np.uint16) if keep_outputs else None
            report.completions.append(Completion(i, requests[i].arrival_s, admitted, done,
                                                 counters, output))
            report.megapixels += int(d_out.shape[0]) * int(d_out.shape[1]) / 1e6
            finished.append(ticket)
        if not finished:
            time.sleep(0.0002)
    report.wall_s = now()
    report.completions.sort(key=lambda c: c.index)
    return report
