"""Host logic of the serving loop (no GPU): arrival schedule and report."""

from __future__ import annotations

import numpy as np

from fauxice_b200 import _lib, serve


def test_poisson_arrivals_are_seeded_sorted_and_bounded():
    a = serve.poisson_arrivals(8.0, 30.0, seed=3)
    b = serve.poisson_arrivals(8.0, 30.0, seed=3)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0) and a.min() >= 0 and a.max() < 30.0
    assert 150 < a.size < 330  # mean 240


def test_report_percentiles_and_throughput():
    report = serve.ServeReport(wall_s=2.0, megapixels=100.0)
    for i, lat in enumerate([0.010, 0.020, 0.030, 0.040]):
        report.completions.append(serve.Completion(i, 1.0, 1.0, 1.0 + lat, _lib.FxCounters()))
    s = report.summary()
    assert s["requests"] == 4 and s["mp_per_s"] == 50.0
    assert s["p50_ms"] == 25.0
    assert s["p50_ms"] <= s["p95_ms"] <= s["p99_ms"] <= 40.0


def test_slot_model_reuses_grows_and_releases_like_the_library():
    model = serve.SlotModel(2)
    assert model.choose(100) == ("new", 0, 100)
    model.take(("new", 0, 100))
    assert model.take(model.choose(300)) == 300
    assert model.allocated == 400 and model.empty == 0
    assert model.choose(50) is None  # both slots busy
    model.give_back(300)
    model.give_back(100)
    assert model.choose(50) == ("reuse", 100, 100)  # the smallest that holds it
    assert model.choose(200) == ("reuse", 300, 300)
    grow = model.choose(400)  # nothing holds it, no empty slot: the largest grows
    assert grow == ("grow", 300, 400) and model.extra(grow) == 100
    model.take(grow)
    assert model.allocated == 500 and model.free_sizes == [100]
    model.release_idle()
    assert model.allocated == 400 and model.empty == 1 and model.free_sizes == []


class FakeDevice:
    """A host-only stand-in for serve.TorchDevice: passes finish after a few
    polls, and the library's slot choice (fx_api free_slot: smallest buffers
    that hold the frame, else a slot without buffers, else grow the largest
    idle one) is replayed to track the device memory the slots hold."""

    def __init__(self, slots: int, polls: int = 3, free: int = 1 << 40):
        self.arena = [0] * slots        # buffer bytes per library slot (0: none)
        self.busy = [False] * slots
        self.polls, self.free = polls, free
        self.peak = 0
        self.grows = 0
        self.passes: dict[int, dict] = {}
        self.next_ticket = 1

    def frame_bytes(self, h, w):
        return 1000 + 20 * h * w

    def free_bytes(self):
        return self.free

    def release_idle(self):
        for k, busy in enumerate(self.busy):
            if not busy:
                self.arena[k] = 0

    def reserve(self, count, h, w, buffers):
        for k in range(count):
            self.arena[k] = max(self.arena[k], self.frame_bytes(h, w))
        self.peak = max(self.peak, sum(self.arena))

    def upload(self, st, pixels):
        st["left"] = self.polls

    def landed(self, st):
        st["left"] -= 1
        return st["left"] <= 0

    def submit(self, st):
        need = self.frame_bytes(st["h"], st["w"])
        idle = [k for k in range(len(self.busy)) if not self.busy[k]]
        if not idle:
            return None
        fits = [k for k in idle if self.arena[k] >= need]
        empty = [k for k in idle if self.arena[k] == 0]
        if fits:
            k = min(fits, key=lambda j: self.arena[j])
        elif empty:
            k = empty[0]
            self.arena[k] = need
        else:
            k = max(idle, key=lambda j: self.arena[j])
            self.arena[k] = need
            self.grows += 1
        self.busy[k] = True
        self.peak = max(self.peak, sum(self.arena))
        ticket, self.next_ticket = self.next_ticket, self.next_ticket + 1
        self.passes[ticket] = {"slot": k, "left": self.polls, "st": st}
        return ticket

    def done(self, ticket):
        self.passes[ticket]["left"] -= 1
        return self.passes[ticket]["left"] <= 0

    def finish(self, ticket):
        p = self.passes.pop(ticket)
        self.busy[p["slot"]] = False
        c = _lib.FxCounters()
        c.attempted = p["st"]["h"] * p["st"]["w"]
        return c

    def download(self, st, expected):
        st["left"] = 1

    def downloaded(self, st):
        st["left"] -= 1
        return st["left"] <= 0

    def output(self, st):
        return np.full((st["h"], st["w"], 3), st["i"], np.uint16)

    def mismatches(self):
        return 0


def _fake_requests(sizes, spacing=0.0):
    return [serve.Request(k * spacing, np.zeros((h, w, 4), np.uint16))
            for k, (h, w) in enumerate(sizes)]


def test_loop_serves_every_request_in_order_within_the_budget():
    rng = np.random.default_rng(4)
    sizes = [(int(h), int(w)) for h, w in rng.integers(8, 300, size=(60, 2))]
    dev = FakeDevice(4)
    largest = max(dev.frame_bytes(h, w) + 14 * h * w for h, w in sizes)
    budget = 2 * largest + largest // 2
    report = serve.serve(None, _fake_requests(sizes, 0.0002), max_slots=4,
                         budget_bytes=budget, keep_outputs=True, device=dev)
    assert [c.index for c in report.completions] == list(range(len(sizes)))
    for c, (h, w) in zip(report.completions, sizes):
        assert c.counters.attempted == h * w and c.output.shape == (h, w, 3)
        assert np.all(c.output == c.index)
    assert report.peak_bytes <= budget
    assert dev.peak <= budget  # the library's slot buffers never exceeded it
    assert report.max_in_flight <= 4


def test_a_large_request_after_small_ones_is_admitted():
    """Every slot holds small buffers and nothing is in flight when a large
    frame arrives: the loop releases the idle buffers instead of waiting."""

    dev = FakeDevice(3)
    sizes = [(10, 10), (12, 12), (14, 14), (200, 200), (11, 11)]
    largest = dev.frame_bytes(200, 200) + 14 * 200 * 200
    report = serve.serve(None, _fake_requests(sizes), max_slots=3, budget_bytes=largest + 5000,
                         warm_slots=0, device=dev)
    assert [c.index for c in report.completions] == list(range(5))
    assert report.releases >= 1 and dev.grows == 0
    assert dev.peak <= largest + 5000


def test_a_large_request_grows_an_idle_slot_when_the_budget_allows():
    dev = FakeDevice(2)
    sizes = [(10, 10), (12, 12), (100, 100)]
    report = serve.serve(None, _fake_requests(sizes, 0.01), max_slots=2,
                         budget_bytes=1 << 30, warm_slots=0, device=dev)
    assert [c.index for c in report.completions] == [0, 1, 2]
    assert report.releases == 0 and dev.grows == 1


def test_warm_slots_are_sized_for_the_largest_request():
    dev = FakeDevice(4)
    sizes = [(10, 10), (100, 100), (20, 20), (100, 100), (50, 50)]
    report = serve.serve(None, _fake_requests(sizes, 0.001), max_slots=4,
                         budget_bytes=1 << 30, warm_slots=2, device=dev)
    assert [c.index for c in report.completions] == list(range(5))
    big = dev.frame_bytes(100, 100)
    assert sorted(dev.arena)[-2:] == [big, big]
    assert dev.grows == 0


def test_a_blocking_device_call_is_reported_and_gc_is_restored():
    """A device call that blocks the single-threaded loop shows up in the
    report (slowest call per kind, calls over 20 ms); the loop runs without
    cyclic garbage collection and turns it back on afterwards."""

    import gc
    import time

    class SlowSubmit(FakeDevice):
        def __init__(self, slots):
            super().__init__(slots)
            self.slow_once = True

        def submit(self, st):
            if self.slow_once:
                self.slow_once = False
                time.sleep(0.03)
            return super().submit(st)

    dev = SlowSubmit(2)
    sizes = [(10, 10), (12, 12), (14, 14)]
    assert gc.isenabled()
    report = serve.serve(None, _fake_requests(sizes, 0.001), max_slots=2,
                         budget_bytes=1 << 30, warm_slots=0, device=dev)
    assert gc.isenabled()
    summary = report.summary()
    assert summary["calls_over_20ms"] >= 1
    assert summary["slowest_call_ms"]["submit"] >= 20.0
    assert summary["longest_stalls"][0][1] == "submit"
    assert summary["capacity_reruns"] == 0
