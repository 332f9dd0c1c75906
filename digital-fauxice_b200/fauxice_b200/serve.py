"""Serving: requests of mixed sizes admitted as they arrive (continuous batching).

No counterpart in the reference.  A request is one RGBI frame in host
memory.  Device memory is sized once, before the run, for the largest
request: every library slot (fx_reserve_frames) and one input/output buffer
pair per slot; the run fails up front with MemoryError when free HBM cannot
hold them.  The loop admits requests in arrival order while a buffer pair is
free, so frames that arrive while others run are processed alongside them:
each upload is queued on a copy stream, the frame is submitted with
fx_submit_device once its upload has landed, and completions are polled.
Latency runs from arrival to the moment the completion is seen.  Results
equal one-frame processing: every request is an independent job.

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
    """Run the request loop in real time; requests must be sorted by arrival.

    Before the clock starts, every library slot is sized for the largest
    request (fx_reserve_frames) and each of ``slots`` device buffer pairs
    (input RGBI, output RGB16) is allocated at that size, so nothing is
    allocated or freed while frames are in flight.  A request is admitted as
    soon as a buffer pair is free: its upload is queued on a copy stream and
    the frame is submitted when the upload's event has completed, so the loop
    never blocks on a copy and keeps polling arrivals and completions.
    """

    import torch

    lib = _lib.load()
    report = ServeReport()
    if not requests:
        return report
    batch.set_slots(ctx, slots)
    max_h = max(int(r.pixels.shape[0]) for r in requests)
    max_w = max(int(r.pixels.shape[1]) for r in requests)
    batch.reserve_frames(ctx, max_h, max_w)
    pair_bytes = slots * max_h * max_w * 14
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    with ctx.lock:
        if (lib.fx_mem_info(ctx.handle, ctypes.byref(free), ctypes.byref(total)) == 0
                and free.value < pair_bytes + reserve_bytes):
            raise MemoryError(f"{slots} buffer pairs for {max_h}x{max_w} frames need "
                              f"{pair_bytes} bytes; {free.value} are free")
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    ins = [torch.empty(max_h * max_w * 4, dtype=torch.int16, device="cuda") for _ in range(slots)]
    outs = [torch.empty(max_h * max_w * 3, dtype=torch.int16, device="cuda") for _ in range(slots)]
    free_pairs: deque[int] = deque(range(slots))
    copy_stream = torch.cuda.Stream()
    waiting: deque[int] = deque()
    staging: deque[tuple] = deque()  # (index, pair, event, admitted): uploads in flight, in order
    inflight: dict[int, tuple] = {}  # ticket -> (index, admitted, pair)
    torch.cuda.synchronize()
    nxt = 0
    start = time.perf_counter()

    def now() -> float:
        return time.perf_counter() - start

    while nxt < len(requests) or waiting or staging or inflight:
        t = now()
        while nxt < len(requests) and requests[nxt].arrival_s <= t:
            waiting.append(nxt)
            nxt += 1
        # admission: a free buffer pair takes the next request's upload
        while waiting and free_pairs:
            i = waiting.popleft()
            pair = free_pairs.popleft()
            src = requests[i].pixels
            if isinstance(src, np.ndarray):
                src = torch.from_numpy(np.ascontiguousarray(src, dtype=np.uint16).view(np.int16))
            h, w = int(src.shape[0]), int(src.shape[1])
            with torch.cuda.stream(copy_stream):
                ins[pair][: h * w * 4].view(h, w, 4).copy_(src, non_blocking=True)
                done = torch.cuda.Event()
                done.record(copy_stream)
            staging.append((i, pair, done, now()))
        # submission: uploads that have landed go to a library slot
        while staging and staging[0][2].query():
            i, pair, _, admitted = staging[0]
            src = requests[i].pixels
            h, w = int(src.shape[0]), int(src.shape[1])
            ticket = ctypes.c_int64()
            with ctx.lock:
                status = lib.fx_submit_device(
                    ctx.handle, ctypes.c_void_p(ins[pair].data_ptr()), h, w,
                    ctypes.byref(params), None, NIKON_PE_INITIAL_STATE,
                    ctypes.c_void_p(outs[pair].data_ptr()), None, None, ctypes.byref(ticket))
            if status == batch.FX_PENDING:
                break
            batch._check(ctx, status)
            staging.popleft()
            inflight[ticket.value] = (i, admitted, pair)
        # completions
        finished = False
        for ticket in list(inflight):
            with ctx.lock:
                status = lib.fx_poll(ctx.handle, ticket)
            if status == batch.FX_PENDING:
                continue
            counters = _lib.FxCounters()
            status = lib.fx_wait(ctx.handle, ticket, -1, ctypes.byref(counters))
            batch._check(ctx, status)
            done_t = now()
            i, admitted, pair = inflight.pop(ticket)
            h, w = (int(v) for v in requests[i].pixels.shape[:2])
            output = None
            if keep_outputs:
                output = outs[pair][: h * w * 3].view(h, w, 3).cpu().numpy().view(np.uint16)
            free_pairs.append(pair)
            report.completions.append(Completion(i, requests[i].arrival_s, admitted, done_t,
                                                 counters, output))
            report.megapixels += h * w / 1e6
            finished = True
        if not finished:
            time.sleep(0.0001)
    report.wall_s = now()
    report.completions.sort(key=lambda c: c.index)
    return report
