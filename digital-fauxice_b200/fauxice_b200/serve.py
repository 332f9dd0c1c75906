"""Serving: requests of mixed sizes admitted as they arrive (continuous batching).

No counterpart in the reference, which processes one job per call.  A
request is one RGBI frame in host memory.  The loop admits requests in
arrival order while the device has room for them, so frames that arrive
while others run are processed alongside them, each in its own library slot
(its own stream and device buffers):

* admission is by device memory: a request needs its pass buffers
  (``fx_pass_bytes(h, w)``: ``fx_frame_bytes``, the same estimate the
  reference's CUDA backend checks against free memory,
  cuda_backend/engine.py:168-224, with the RNG-dependent list grown by any
  overflow the context has seen) plus its input and output planes.  A slot whose buffers already hold the frame is reused
  (no new memory); otherwise a slot without buffers takes it, or the idle
  slot with the largest buffers grows, if the bytes fit the budget (the
  free HBM reported by ``fx_mem_info`` at the start, less a reserve).  When
  a request does not fit while nothing is in flight, the idle slots'
  buffers are released (``fx_release_idle_slots``; freeing device memory
  waits for the whole device, which costs nothing then) and the request is
  admitted into fresh ones.
* a request's upload is queued on a copy stream; the frame is submitted
  with ``fx_submit_device`` once the upload has landed; when the pass is
  done its RGB16 output is copied back into pinned host memory on a second
  copy stream.  The loop never blocks on a copy.
* latency runs from arrival to the moment the output is in host memory.
* optionally, each output is compared on the device, bit for bit, with the
  output of the same frame processed alone (kept resident for the check);
  the count of differing values is read once, after the run.

Device memory for inputs and outputs is plumbing (torch tensors from its
caching allocator); the processing itself is the library's.
"""

from __future__ import annotations

import ctypes
import gc
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
    expected: object = None  # the frame's RGB16 output processed alone: a
                             # device int16 tensor (H, W, 3), for verification


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

    @property
    def queued_s(self) -> float:
        return self.admitted_s - self.arrival_s


@dataclass
class ServeReport:
    completions: list[Completion] = field(default_factory=list)
    wall_s: float = 0.0
    megapixels: float = 0.0
    max_in_flight: int = 0
    peak_bytes: int = 0        # slot buffers + planes of the requests in flight
    budget_bytes: int = 0
    slots_used: int = 0        # library slots that got device buffers
    releases: int = 0          # times the idle slots' buffers were released
    verified: int = 0          # outputs compared with their single-frame output
    mismatches: int = 0        # differing uint16 values over all verified outputs
    slowest_call_s: dict = field(default_factory=dict)  # device call -> longest host time
    stalls: list = field(default_factory=list)  # (at_s, call, ms, in flight) of calls > 20 ms

    def note_call(self, name: str, seconds: float, at_s: float = 0.0, in_flight: int = 0) -> None:
        if seconds > self.slowest_call_s.get(name, 0.0):
            self.slowest_call_s[name] = seconds
        if seconds > 0.020:
            self.stalls.append((round(at_s, 3), name, round(seconds * 1e3, 1), in_flight))

    def percentile_ms(self, q: float, attr: str = "latency_s") -> float:
        lat = np.array([getattr(c, attr) for c in self.completions]) * 1e3
        return float(np.percentile(lat, q)) if lat.size else float("nan")

    def summary(self) -> dict:
        out = {"requests": len(self.completions), "wall_s": round(self.wall_s, 3),
               "mp_per_s": round(self.megapixels / self.wall_s, 1) if self.wall_s else None,
               "p50_ms": round(self.percentile_ms(50), 2),
               "p95_ms": round(self.percentile_ms(95), 2),
               "p99_ms": round(self.percentile_ms(99), 2),
               "queue_p50_ms": round(self.percentile_ms(50, "queued_s"), 2),
               "queue_p99_ms": round(self.percentile_ms(99, "queued_s"), 2),
               "max_in_flight": self.max_in_flight,
               "peak_device_bytes": self.peak_bytes,
               "budget_bytes": self.budget_bytes,
               "slots_used": self.slots_used,
               "buffer_releases": self.releases,
               "capacity_reruns": int(sum(getattr(c.counters, "capacity_reruns", 0)
                                          for c in self.completions)),
               "slowest_call_ms": {k: round(v * 1e3, 2)
                                   for k, v in sorted(self.slowest_call_s.items())},
               "calls_over_20ms": len(self.stalls),
               "longest_stalls": sorted(self.stalls, key=lambda x: -x[2])[:5]}
        if self.verified:
            out["verified"] = self.verified
            out["bit_exact"] = self.mismatches == 0 and self.verified == len(self.completions)
        return out


def poisson_arrivals(rate_per_s: float, duration_s: float, seed: int) -> np.ndarray:
    """Arrival times of a seeded Poisson process on [0, duration)."""

    rng = np.random.default_rng(seed)
    times, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate_per_s)
        if t >= duration_s:
            return np.array(times)
        times.append(t)


def frame_bytes(height: int, width: int) -> int:
    """Device bytes of one pass's buffers (fx_frame_bytes)."""

    return int(_lib.load().fx_frame_bytes(int(height), int(width)))


class SlotModel:
    """The library's slot choice (fx_api free_slot), mirrored on the host:
    the idle slot with the smallest buffers that hold the frame, else a slot
    without buffers, else the idle slot with the largest buffers, which
    grows.  Tracks the buffer sizes so admission knows how much new device
    memory a request needs."""

    def __init__(self, slots: int) -> None:
        self.free_sizes: list[int] = []   # buffers of idle slots
        self.empty = slots                 # slots without buffers
        self.allocated = 0                 # bytes of all slot buffers

    def choose(self, need: int) -> tuple[str, int, int] | None:
        """(kind, old buffer size, new buffer size), or None when every slot
        is busy."""

        fits = [s for s in self.free_sizes if s >= need]
        if fits:
            return "reuse", min(fits), min(fits)
        if self.empty:
            return "new", 0, need
        if self.free_sizes:
            return "grow", max(self.free_sizes), need
        return None

    @staticmethod
    def extra(choice: tuple[str, int, int]) -> int:
        kind, old, new = choice
        return 0 if kind == "reuse" else new - old

    def take(self, choice: tuple[str, int, int]) -> int:
        """Mark the chosen slot busy; returns its buffer size."""

        kind, old, new = choice
        if kind == "reuse":
            self.free_sizes.remove(old)
        elif kind == "new":
            self.empty -= 1
            self.allocated += new
        else:
            self.free_sizes.remove(old)
            self.allocated += new - old
        return new

    def give_back(self, size: int) -> None:
        self.free_sizes.append(size)

    def release_idle(self) -> None:
        """The idle slots' buffers were freed."""

        self.empty += len(self.free_sizes)
        self.allocated -= sum(self.free_sizes)
        self.free_sizes = []


class TorchDevice:
    """The device side of the request loop: torch streams and buffers for
    the planes and the copies, the library for the passes."""

    def __init__(self, ctx: _lib.Context, max_slots: int, max_out: int) -> None:
        import torch

        self.torch = torch
        self.ctx = ctx
        self.lib = _lib.load()
        self.params = DEFAULT_PROFILE.hot_path_parameters().to_c()
        batch.set_slots(ctx, max_slots)
        self.host_out = [torch.empty(max_out, dtype=torch.int16).pin_memory()
                         for _ in range(max_slots)]
        self.up, self.down, self.checks = (torch.cuda.Stream(), torch.cuda.Stream(),
                                           torch.cuda.Stream())
        self.mismatch = torch.zeros((), dtype=torch.int64, device="cuda")
        # the loop's own device work once, before any clock: the first launch
        # of a kernel loads its module (lazy loading), about 0.1 s
        n = min(96, max_out)
        probe = torch.zeros(n, dtype=torch.int16, device="cuda")
        with torch.cuda.stream(self.checks):
            self.mismatch.add_((probe != probe).sum())
        with torch.cuda.stream(self.down):
            self.host_out[0][:n].copy_(probe, non_blocking=True)
        with torch.cuda.stream(self.up):
            probe.copy_(self.host_out[0][:n], non_blocking=True)
        torch.cuda.synchronize()

    def frame_bytes(self, h: int, w: int) -> int:
        """Pass buffers of an h x w frame on this context (fx_pass_bytes:
        the list grown by any overflow the context has seen)."""

        out = ctypes.c_int64()
        with self.ctx.lock:
            self.ctx.check(self.lib.fx_pass_bytes(self.ctx.handle, h, w, ctypes.byref(out)))
        return int(out.value)

    def free_bytes(self) -> int:
        free, total = ctypes.c_size_t(), ctypes.c_size_t()
        with self.ctx.lock:
            self.ctx.check(self.lib.fx_mem_info(self.ctx.handle, ctypes.byref(free),
                                                ctypes.byref(total)))
        return int(free.value)

    def release_idle(self) -> None:
        with self.ctx.lock:
            self.ctx.check(self.lib.fx_release_idle_slots(self.ctx.handle, None))

    def reserve(self, count: int, h: int, w: int, buffers: int) -> None:
        """Before the clock: size ``count`` slots for an h x w frame, and
        let torch's caching allocator hold ``buffers`` input/output pairs of
        that size, so the loop allocates no device memory for them."""

        torch = self.torch
        with self.ctx.lock:
            self.ctx.check(self.lib.fx_reserve_slots(self.ctx.handle, count, h, w))
        with torch.cuda.stream(self.up):
            held = [(torch.empty((h, w, 4), dtype=torch.int16, device="cuda"),
                     torch.empty((h, w, 3), dtype=torch.int16, device="cuda"))
                    for _ in range(buffers)]
        del held
        torch.cuda.synchronize()

    def upload(self, st: dict, pixels) -> None:
        torch = self.torch
        h, w = st["h"], st["w"]
        src = pixels
        if isinstance(src, np.ndarray):
            src = torch.from_numpy(np.ascontiguousarray(src, dtype=np.uint16).view(np.int16))
        with torch.cuda.stream(self.up):
            st["d_in"] = torch.empty((h, w, 4), dtype=torch.int16, device="cuda")
            st["d_out"] = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
            st["d_in"].copy_(src.view(h, w, 4), non_blocking=True)
            st["event"] = torch.cuda.Event()
            st["event"].record(self.up)

    def landed(self, st: dict) -> bool:
        return st["event"].query()

    def submit(self, st: dict) -> int | None:
        ticket = ctypes.c_int64()
        with self.ctx.lock:
            status = self.lib.fx_submit_device(
                self.ctx.handle, ctypes.c_void_p(st["d_in"].data_ptr()), st["h"], st["w"],
                ctypes.byref(self.params), None, NIKON_PE_INITIAL_STATE,
                ctypes.c_void_p(st["d_out"].data_ptr()), None, None, ctypes.byref(ticket))
        if status == batch.FX_PENDING:
            return None
        batch._check(self.ctx, status)
        return ticket.value

    def done(self, ticket: int) -> bool:
        with self.ctx.lock:
            return self.lib.fx_poll(self.ctx.handle, ticket) != batch.FX_PENDING

    def finish(self, ticket: int) -> _lib.FxCounters:
        counters = _lib.FxCounters()
        batch._check(self.ctx, self.lib.fx_wait(self.ctx.handle, ticket, -1,
                                                ctypes.byref(counters)))
        return counters

    def download(self, st: dict, expected) -> None:
        """Queue the output's copy to pinned host memory and, when given,
        its on-device comparison (the pass is complete: fx_wait returned)."""

        torch = self.torch
        n = st["h"] * st["w"] * 3
        with torch.cuda.stream(self.down):
            self.host_out[st["host"]][:n].copy_(st["d_out"].view(-1), non_blocking=True)
            st["event"] = torch.cuda.Event()
            st["event"].record(self.down)
        if expected is not None:
            with torch.cuda.stream(self.checks):
                self.mismatch.add_((st["d_out"] != expected.view(st["h"], st["w"], 3)).sum())
            st["d_out"].record_stream(self.checks)

    def downloaded(self, st: dict) -> bool:
        return st["event"].query()

    def output(self, st: dict) -> np.ndarray:
        n = st["h"] * st["w"] * 3
        return self.host_out[st["host"]][:n].numpy().view(np.uint16).reshape(
            st["h"], st["w"], 3).copy()

    def mismatches(self) -> int:
        self.checks.synchronize()
        return int(self.mismatch.item())


def serve(ctx: _lib.Context | None, requests: Sequence[Request], *, max_slots: int = 12,
          budget_bytes: int | None = None, reserve_bytes: int = 8 << 30,
          keep_outputs: bool = False, warm_slots: int = 4, device=None) -> ServeReport:
    """Run the request loop in real time; requests must be sorted by arrival.

    ``max_slots`` bounds the requests in flight; device memory bounds them
    too: ``budget_bytes`` (default: the free HBM at the start less
    ``reserve_bytes``) must hold every slot's buffers plus the input and
    output planes of the requests in flight.  A request that carries its
    ``expected`` output is checked against it on the device, after its
    output's copy to host memory has been queued (off the latency path).
    The idle slots' buffers are released before the clock starts, so the
    host's model of the slots and the library's slots start out empty; then
    ``warm_slots`` slots are sized for the largest request (as far as the
    budget allows), so the first requests find buffers ready.
    ``device`` replaces the device side (a :class:`TorchDevice` on ``ctx``
    by default; the tests drive the loop with a host-only stand-in).
    """

    report = ServeReport()
    if not requests:
        return report
    max_out = max(int(r.pixels.shape[0]) * int(r.pixels.shape[1]) * 3 for r in requests)
    dev = device if device is not None else TorchDevice(ctx, max_slots, max_out)
    dev.release_idle()  # nothing is in flight yet: start from slots without buffers
    if budget_bytes is None:
        budget_bytes = dev.free_bytes() - reserve_bytes
    report.budget_bytes = int(budget_bytes)
    largest = max(dev.frame_bytes(*r.pixels.shape[:2]) + 14 * int(r.pixels.shape[0])
                  * int(r.pixels.shape[1]) for r in requests)
    if largest > budget_bytes:
        raise MemoryError(f"the largest request needs {largest} bytes of device memory; the "
                          f"budget is {budget_bytes}")
    model = SlotModel(max_slots)
    big = max(requests, key=lambda r: dev.frame_bytes(*r.pixels.shape[:2]))
    bh, bw = (int(v) for v in big.pixels.shape[:2])
    big_bytes = dev.frame_bytes(bh, bw)
    warm = min(warm_slots, max_slots, max(0, (budget_bytes - 14 * bh * bw) // big_bytes))
    if warm > 0:
        dev.reserve(warm, bh, bw, max_slots)
        model.free_sizes = [big_bytes] * warm
        model.empty -= warm
        model.allocated += warm * big_bytes
    free_host = deque(range(max_slots))
    waiting: deque[int] = deque()
    staging: deque[dict] = deque()    # uploads in flight, in admission order
    inflight: dict[int, dict] = {}    # ticket -> request state
    downloads: deque[dict] = deque()  # outputs on their way to host memory
    in_use_bytes = 0                  # planes of the requests in flight
    nxt = 0
    # no cyclic garbage collection while requests are timed: a full
    # collection over a large process heap pauses the loop for tens of
    # milliseconds, and every request in flight waits for it
    collect = gc.isenabled()
    gc.collect()
    gc.disable()
    try:
        start = time.perf_counter()

        def now() -> float:
            return time.perf_counter() - start

        def call(name: str, fn, *args):
            """A device call of the loop, with its host time noted: the loop is
            single-threaded, so a call that blocks delays every request."""

            t0 = time.perf_counter()
            out = fn(*args)
            report.note_call(name, time.perf_counter() - t0, t0 - start,
                             len(staging) + len(inflight) + len(downloads))
            return out

        while nxt < len(requests) or waiting or staging or inflight or downloads:
            t = now()
            while nxt < len(requests) and requests[nxt].arrival_s <= t:
                waiting.append(nxt)
                nxt += 1
            # admission, in arrival order: a slot (reused, new or grown) and room
            while waiting and free_host:
                i = waiting[0]
                h, w = (int(v) for v in requests[i].pixels.shape[:2])
                planes = 14 * h * w
                choice = model.choose(dev.frame_bytes(h, w))
                fits = (choice is not None and model.allocated + model.extra(choice) + in_use_bytes
                        + planes <= budget_bytes)
                if not fits:
                    if staging or inflight or downloads or not model.free_sizes:
                        break  # wait for a request in flight to finish
                    # nothing in flight: drop the idle buffers and start afresh
                    call("release_idle", dev.release_idle)
                    model.release_idle()
                    report.releases += 1
                    continue
                waiting.popleft()
                st = {"i": i, "h": h, "w": w, "admitted": now(), "size": model.take(choice),
                      "planes": planes, "host": free_host.popleft()}
                in_use_bytes += planes
                call("upload", dev.upload, st, requests[i].pixels)
                staging.append(st)
            report.max_in_flight = max(report.max_in_flight,
                                       len(staging) + len(inflight) + len(downloads))
            report.peak_bytes = max(report.peak_bytes, model.allocated + in_use_bytes)
            # submission: uploads that have landed go to a library slot
            while staging and dev.landed(staging[0]):
                ticket = call("submit", dev.submit, staging[0])
                if ticket is None:
                    break
                inflight[ticket] = staging.popleft()
            # finished passes: counters, then the output's copy to host memory
            for ticket in list(inflight):
                if not call("poll", dev.done, ticket):
                    continue
                st = inflight.pop(ticket)
                st["counters"] = call("finish", dev.finish, ticket)
                expected = requests[st["i"]].expected
                call("download", dev.download, st, expected)
                if expected is not None:
                    report.verified += 1
                downloads.append(st)
            finished = False
            while downloads and dev.downloaded(downloads[0]):
                st = downloads.popleft()
                done_t = now()
                i, h, w = st["i"], st["h"], st["w"]
                output = dev.output(st) if keep_outputs else None
                free_host.append(st["host"])
                model.give_back(st["size"])
                in_use_bytes -= st["planes"]
                report.completions.append(Completion(i, requests[i].arrival_s, st["admitted"],
                                                     done_t, st["counters"], output))
                report.megapixels += h * w / 1e6
                finished = True
            if not finished:
                time.sleep(0.0001)
        report.wall_s = now()
    finally:
        if collect:
            gc.enable()
    report.slots_used = max_slots - model.empty
    report.mismatches = dev.mismatches()
    report.completions.sort(key=lambda c: c.index)
    return report
