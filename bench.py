#!/usr/bin/env python3
"""Headline benchmark: bit-exact full-frame megapixels/s on B200.

One step = the whole Digital ICE main pass over one native 4000 dpi frame
(5782x3946 RGBI uint16, seeded synthetic generator, defects on ~6% of the
pixels): device producer schedule and stage table, planes, 9x9 stencil,
hidden startup replay, dither writer, emit and counters.

  value  device-resident input and output (HBM), CUDA events on the launch
         stream, max over ranks; MP/s of the whole job.
  e2e    the public API a user calls, process_b200(job) -> ProcessingResult,
         host buffers in and out (H2D of the RGBI frame, D2H of the RGB16
         output, output SHA-256) timed per call.
  --impl reference  times the CPU restatement of the reference path
         (oracle/, OpenMP over all host cores) on the same workload.

Multi-GPU: one process per GPU.  Under torchrun the ranks come from the
environment; ``--gpus N`` without one relaunches this script under
torch.distributed.run itself.  Rank r processes its own frame (seed 2 + r;
frames are independent jobs), with no collective on the data path: the
only collectives are the barriers around the timed region and the maximum
of the ranks' elapsed times.  ``--plan-only`` prints the per-rank work plan
after those collectives and exits (no GPU work; gloo on a CPU machine).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import socket
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "digital-fauxice_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = ("bit-exact full-frame megapixels/s on 1 B200 (batched vs plain); "
          "p50/p99 frame latency")
HEIGHT, WIDTH = 5782, 3946
SEED = 2
# Algorithmic bytes: the stencil stage reads 8 B of
# RGBI and writes a 24 B float64 candidate plus 1 B of status per pixel; the
# serial walk reads a 32 B interval/jump entry and writes a 4 B running count
# per RNG-dependent channel.
STENCIL_BYTES_PER_PIXEL = 33
WALK_BYTES_PER_CHANNEL = 36
BATCH_FRAMES = 16          # uneven sizes, seeds 100..115
HEAVY_FRAMES = 8           # full 5782x3946 frames at ~5% coverage, seeds 200..207
SERVE_RATES = (2.0, 8.0, 32.0, 400.0)  # the last one above the GPU's capacity
# DRAM bytes and warp instructions per k_stencil launch from an ncu capture
NCU_COUNTERS = os.path.join(ROOT, "profiles", "ncu_counters.json")


WALK_BLOCKS_PER_SM = 3   # window-walk blocks per SM in one wave (kWinBlocksPerSM)


def launches_per_frame(h: int, w: int, sms: int) -> int:
    """Kernel launches of one plain pass (the library's launch sequence):
    producer 3, planes 1, stencil 1, startup 1, chain 4, walk 1 per wave + 1
    rewalk, apply 3.  Waves are sized from the RNG-dependent list capacity,
    with three window blocks per SM less one slot for the wave's resolve
    block."""

    sites = 6 * w + h * w
    capacity = max(65536, sites // 2)
    segments = (capacity + 4095) // 4096 + 1
    per_wave = WALK_BLOCKS_PER_SM * sms - 1
    waves = (segments + per_wave - 1) // per_wave
    return 14 + waves


def ncu_counter(kernel: str, name: str):
    """A counter of one kernel's committed ncu capture (None if absent)."""

    try:
        with open(NCU_COUNTERS) as handle:
            return json.load(handle)[kernel][name]
    except (OSError, KeyError, ValueError):
        return None


def stencil_traffic():
    return ncu_counter("k_stencil", "dram_bytes_per_launch")


def issue_roofline(stencil_ms: float, device: int):
    """The stencil's second bound: it is instruction-bound (binary64 chains in
    the reference's operation order), so its warp instructions per launch
    over its CUDA-event time are compared with the SMs' peak issue rate (four
    warp instructions per SM per cycle at the maximum SM clock)."""

    import torch

    inst = stencil_warp_instructions()
    if inst is None or stencil_ms <= 0:
        return None
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    try:
        mhz = float(subprocess.run(
            ["nvidia-smi", "-i", str(device), "--query-gpu=clocks.max.sm",
             "--format=csv,noheader,nounits"], capture_output=True, text=True,
            timeout=10).stdout.strip().splitlines()[0])
    except (OSError, ValueError, IndexError, subprocess.SubprocessError):
        mhz = 1965.0
    achieved = inst / (stencil_ms / 1000.0) / 1e9
    peak = 4.0 * sms * mhz / 1000.0
    return {"bound": "issue", "warp_instructions_per_launch": inst,
            "achieved": round(achieved, 1), "peak": round(peak, 1), "unit": "G warp-inst/s",
            "frac": round(achieved / peak, 4),
            "source": "instructions from the ncu capture in profiles/ncu_counters.json, "
                      "time from this run's CUDA events, peak = 4 x SMs x max SM clock"}


def stencil_warp_instructions():
    value = ncu_counter("k_stencil", "warp_instructions_per_launch")
    return float(value) if value is not None else None


def _batch_frame(index: int):
    for _p in (ROOT, os.path.join(ROOT, "digital-fauxice_b200")):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    from fauxice_b200 import synthetic

    return synthetic.batch_frame(index)[0]


def _heavy_frame(index: int):
    for _p in (ROOT, os.path.join(ROOT, "digital-fauxice_b200")):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    from fauxice_b200 import synthetic

    return synthetic.heavy_full_frame(index)[0]


def _serving_frame(spec):
    for _p in (ROOT, os.path.join(ROOT, "digital-fauxice_b200")):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    from fauxice_b200 import synthetic

    seed, h, w, coverage = spec
    return synthetic.coverage_frame(seed, h, w, coverage)


def generate(fn, items):
    """Frames generated in spawn workers (before any CUDA call here)."""

    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(len(items), os.cpu_count() or 1)) as pool:
        return pool.map(fn, items)


def serving_pool_specs(seed: int = 500):
    """The serving pool: 4 full frames, 4 of 2892x1973 and 8 crops of
    U[256, 2048]^2, each with its own defect coverage drawn from
    U[0.1%, 3%] (seed, height, width, coverage)."""

    rng = np.random.default_rng(seed)
    specs = []
    for k, (h, w) in enumerate([(5782, 3946)] * 4 + [(2892, 1973)] * 4):
        specs.append((seed + k, h, w, float(rng.uniform(0.001, 0.03))))
    for k in range(8):
        h, w = (int(v) for v in rng.integers(256, 2049, size=2))
        specs.append((seed + 8 + k, h, w, float(rng.uniform(0.001, 0.03))))
    return specs


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference", "numba"), default="b200",
                    help="reference: the CPU restatement of the path on all host cores; numba: "
                         "the reference's own cpu-fast backend, when installed in baseline/_ref")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-routing", action="store_true",
                    help="skip the at-floor routing census measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and serving runs")
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--no-heavy", action="store_true", help="skip the heavy-damage batch")
    ap.add_argument("--serve-seconds", type=float, default=6.0,
                    help="arrival window per request rate (the workload's 120 s, shortened)")
    ap.add_argument("--serve-rates", default=",".join(f"{r:g}" for r in SERVE_RATES),
                    help="comma-separated Poisson request rates per second")
    ap.add_argument("--stencil-tile", type=int, default=0,
                    help="stencil tile rows of the plain path (8 or 16; 0: library default)")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving workload and print its report")
    ap.add_argument("--plan-only", action="store_true",
                    help="print each rank's work plan after the collectives; no GPU work")
    return ap.parse_args()


def free_port() -> int:
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def launch_command(gpus: int, argv: list[str], port: int) -> list[str]:
    """This script relaunched as ``gpus`` ranks, one process per GPU."""

    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
            os.path.abspath(__file__), *argv]


def rank_plan(rank: int, world: int) -> dict:
    """What rank ``rank`` processes: its own native frame (seed 2 + rank)
    for the timed plain path."""

    from fauxice_b200 import replicas

    seeds = replicas.shard(list(range(SEED, SEED + world)), rank, world)
    return {"rank": rank, "frame_seeds": seeds}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as handle:
            peaks = json.load(handle)
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
               "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(plan_only: bool = False):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "gloo" if plan_only or not torch.cuda.is_available() else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def run_plan(world: int, rank: int) -> None:
    """The plan of every rank, gathered after the timed region's collectives."""

    plan = rank_plan(rank, world)
    barrier(world)
    slowest = max_over_ranks(0.5 + rank, world)
    plans = [plan]
    if world > 1:
        import torch.distributed as dist

        plans = [None] * world
        dist.all_gather_object(plans, plan)
    if rank == 0:
        print(json.dumps({"world": world, "plans": plans, "max_over_ranks": slowest}),
              flush=True)


def max_over_ranks(value: float, world: int) -> float:
    from fauxice_b200 import replicas

    return replicas.max_over_ranks(value) if world > 1 else value


def barrier(world: int) -> None:
    if world > 1:
        from fauxice_b200 import replicas

        replicas.barrier()


def make_job(main, prepass):
    from fauxice_b200 import contracts

    return contracts.ProcessingJob(
        acquisition=contracts.DualRGBIAcquisition(
            prepass=contracts.RGBI16Frame(prepass, contracts.AcquisitionEpoch.PREPASS, 285, "p"),
            main=contracts.RGBI16Frame(main, contracts.AcquisitionEpoch.MAIN, 4000, "m"),
            same_frame_id="bench"),
        scanner_model=contracts.ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED,
        mode=contracts.ProcessingMode.NORMAL, selector=8, resolution_metric=4000, bit_depth=16,
        focus_exposure_locked=True)


def cpu_reference(main, prepass, steps: int, warmup: int, sample_s: float = 6.0):
    """Time the oracle (C, OpenMP, all host cores) on bounded row bands."""

    from oracle import oracle as ox

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ox.process(main, prepass, threads=cores, diagnostics=False)
    full_s = time.perf_counter() - t0
    rows = main.shape[0]
    if full_s > sample_s:
        rows = max(64, int(main.shape[0] * sample_s / full_s))
    sample = np.ascontiguousarray(main[:rows])
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        ox.process(sample, prepass, threads=cores, diagnostics=False)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    mp = sample.shape[0] * sample.shape[1] / 1e6
    return {
        "value": round(mp * len(times) / sum(times), 4),
        "unit": "MP/s",
        "cores": cores,
        "kind": "port",
        "sample": f"{rows}x{main.shape[1]} rows of the seed-{SEED} native frame per step, "
                  f"{len(times)} steps (full frame {full_s:.2f} s)",
        "seconds_per_step": round(sum(times) / len(times), 3),
    }


def run_reference(args, world, rank):
    if rank != 0:
        return
    from fauxice_b200 import synthetic

    main, prepass = synthetic.native_frame(SEED)
    base = cpu_reference(main, prepass, args.steps, args.warmup)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": base["value"],
        "unit": "MP/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1000.0 * base["seconds_per_step"], 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "native 5782x3946 RGBI frame (seeded generator), CPU "
                               "restatement of the reference path",
                   "parallelism": "host threads"},
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": "MP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_numba(args, world, rank):
    """The reference's own numba backend (fast_cpu/engine.py:537,
    process_cpu_fast) on the seed-2 native frame, on all host cores and on
    one thread, after a warm-up that compiles it.  It runs only where the
    reference is installed in baseline/_ref (pip --target); otherwise the
    line says it is unavailable."""

    if rank != 0:
        return
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "portable_digital_ice")):
        print(json.dumps({"impl": "numba", "unavailable": "the reference is not installed in "
                                                          "baseline/_ref"}), flush=True)
        return
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/fauxice_numba_cache")
    sys.path.insert(0, ref)
    import numba
    from portable_digital_ice import (AcquisitionEpoch, DualRGBIAcquisition, ProcessingJob,
                                      ProcessingMode, RGBI16Frame, ScannerModel)
    from portable_digital_ice.fast_cpu import process_cpu_fast

    from fauxice_b200 import synthetic

    def job(main, prepass):
        return ProcessingJob(
            acquisition=DualRGBIAcquisition(
                prepass=RGBI16Frame(prepass, AcquisitionEpoch.PREPASS, 285, "p"),
                main=RGBI16Frame(main, AcquisitionEpoch.MAIN, 4000, "m"), same_frame_id="n"),
            scanner_model=ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED, mode=ProcessingMode.NORMAL,
            selector=8, resolution_metric=4000, bit_depth=16, focus_exposure_locked=True)

    process_cpu_fast(job(*synthetic.small_crop(1)))  # compile
    main, prepass = synthetic.native_frame(SEED)
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_results.json")))
    expect = golden["jobs"]["native_full"]["output_sha256"]
    mp = main.shape[0] * main.shape[1] / 1e6
    cores = numba.config.NUMBA_NUM_THREADS
    out = {}
    for threads, steps in ((cores, max(1, min(args.steps, 3))), (1, 1)):
        numba.set_num_threads(threads)
        times, ok = [], True
        for _ in range(steps):
            t0 = time.perf_counter()
            res = process_cpu_fast(job(main, prepass))
            times.append(time.perf_counter() - t0)
            ok &= res.replay.output_sha256 == expect
        med = sorted(times)[len(times) // 2]
        out[threads] = {"seconds": [round(t, 3) for t in times], "median_s": round(med, 3),
                        "mp_per_s": round(mp / med, 4), "bit_exact": bool(ok)}
    best = out[cores]
    print(json.dumps({
        "impl": "numba", "metric": METRIC, "value": best["mp_per_s"], "unit": "MP/s",
        "n_gpus": args.gpus, "steps": len(best["seconds"]), "warmup": 1,
        "ms_per_step": round(1000 * best["median_s"], 1), "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "native 5782x3946 RGBI frame (seed 2), the reference's numba "
                               "cpu-fast backend (process_cpu_fast)"},
        "cpu_baseline": {"value": best["mp_per_s"], "unit": "MP/s", "cores": cores,
                         "kind": "reference", "sample": "the whole native frame, warm"},
        "one_thread": out[1], "all_cores": best}), flush=True)


def run_b200(args, world, rank, local, frames=None, heavy=None, pool=None):
    import torch

    from fauxice_b200 import _lib, engine, synthetic
    from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE

    torch.cuda.set_device(local)
    seed = rank_plan(rank, world)["frame_seeds"][0]  # rank r: its own frame, seed 2 + r
    main, prepass = synthetic.native_frame(seed)
    h, w = main.shape[:2]
    lib = _lib.load()
    ctx = engine.context(local)
    ctx.check(lib.fx_set_stencil_tile(ctx.handle, args.stencil_tile))
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    d_in = torch.from_numpy(main.view(np.int16)).to(f"cuda:{local}")
    d_out = torch.empty((h, w, 3), dtype=torch.int16, device=f"cuda:{local}")
    stream = torch.cuda.Stream(device=f"cuda:{local}")  # non-default: events see our work

    def step():
        status = lib.fx_process_device(ctx.handle, d_in.data_ptr(), h, w, ctypes.byref(params),
                                       None, NIKON_PE_INITIAL_STATE, d_out.data_ptr(), None, None,
                                       ctypes.c_void_p(stream.cuda_stream), None)
        ctx.check(status)

    counters = _lib.FxCounters()
    # warm-up (and a parity check of this exact workload against the golden record)
    for _ in range(max(args.warmup, 3)):
        step()
    ctx.check(lib.fx_sync_counters(ctx.handle, ctypes.byref(counters)))
    torch.cuda.synchronize()
    import hashlib

    out_host = d_out.cpu().numpy().view(np.uint16)
    digest = hashlib.sha256(out_host.astype("<u2").tobytes()).hexdigest()
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_results.json")))
    expect = golden["jobs"]["native_full"]  # the seed-2 frame: rank 0's
    bit_exact = (digest == expect["output_sha256"]
                 and counters.attempted == expect["attempted_pixels"]
                 and counters.public_advances == expect["public_rng_advances"]
                 and counters.final_state == expect["final_rng_state"]) if seed == SEED else None

    ctx.check(lib.fx_profile_enable(ctx.handle, 1))
    ctx.check(lib.fx_profile_read(ctx.handle, None, None, 1))
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        uuid = None
    sampler = ClockSampler(uuid)
    events = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    events[0].record(stream)
    for i in range(args.steps):
        step()
        events[i + 1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    per_step = [events[i].elapsed_time(events[i + 1]) for i in range(args.steps)]
    elapsed_ms = events[0].elapsed_time(events[-1])
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    stage_ms = (ctypes.c_double * 7)()
    passes = ctypes.c_int64()
    ctx.check(lib.fx_profile_read(ctx.handle, stage_ms, ctypes.byref(passes), 1))
    ctx.check(lib.fx_profile_enable(ctx.handle, 0))
    ctx.check(lib.fx_sync_counters(ctx.handle, ctypes.byref(counters)))
    stages = {name: stage_ms[i] / max(1, passes.value) for i, name in enumerate(_lib.PROFILE_STAGES)}

    mp = h * w / 1e6
    value = world * args.steps * mp / (elapsed_ms / 1000.0)

    # roofline of the largest single kernel launch (k_stencil): algorithmic
    # bytes of the a1-a10 stage, 33 B per pixel, over its CUDA-event time
    peak, peak_kind = load_peaks()
    bytes_per_launch = STENCIL_BYTES_PER_PIXEL * h * w
    achieved = bytes_per_launch / (stages["stencil"] / 1000.0) / 1e9
    roofline = {
        "kernel": "k_stencil",
        "bound": "hbm",
        "achieved": round(achieved, 2),
        "peak": peak,
        "unit": "GB/s",
        "frac": round(achieved / peak, 5),
        "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                        else "fallback: 6650 GB/s, an earlier copy measurement on this GPU "
                             "type (MEASURED_PEAKS.json absent)"),
        "traffic": stencil_traffic(),
        "algorithmic_bytes_per_launch": bytes_per_launch,
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "issue": issue_roofline(stages["stencil"], local),
        "walk": {"bytes_per_channel": WALK_BYTES_PER_CHANNEL,
                 "achieved_gbs": round(WALK_BYTES_PER_CHANNEL * counters.rng_dependent
                                       / (stages["walk"] / 1000.0) / 1e9, 2),
                 "note": "dependent integer chain (latency-bound), not HBM-bound"},
    }

    # end to end through the public API, host buffers in and out
    e2e = None
    if args.e2e_steps > 0:
        job = make_job(main, prepass)
        engine.process_b200(job)  # warm
        times = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            result = engine.process_b200(job)
            times.append(time.perf_counter() - t0)
        e2e_ok = result.replay.output_sha256 == digest
        e2e_s = max_over_ranks(sum(times) / len(times), world)
        e2e = {"value": round(world * mp / e2e_s, 3), "unit": "MP/s",
               "h2d_bytes_per_step": int(main.nbytes), "d2h_bytes_per_step": int(h * w * 6),
               "ms_per_step": round(1000 * e2e_s, 2), "bit_exact": bool(e2e_ok),
               "api": "fauxice_b200.process_b200(job) (host numpy in/out, output SHA-256)"}

    cpu = None
    if not args.no_cpu_baseline and world == 1 and rank == 0:
        cpu = cpu_reference(main, prepass, steps=1, warmup=0, sample_s=12.0)
        cpu.pop("seconds_per_step", None)

    if rank == 0:
        lat = sorted(per_step)
        line = {
            "metric": METRIC,
            "value": round(value, 3),
            "unit": "MP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(elapsed_ms / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {
                "workload": "plain single-frame path, native 5782x3946 RGBI uint16 frame "
                            "(seed 2 + rank; 3000 discs and 60 scratches touching ~6% of "
                            "the pixels), inputs resident in HBM",
                "frames_per_step": 1,
                "l2": "inputs 182.5 MB per frame > 126 MB L2; no flush",
                "parallelism": f"replicas x{world}",
                "bit_exact_vs_reference": bit_exact,
            },
            "latency_ms": {"p50": round(lat[len(lat) // 2], 3),
                           "p99": round(lat[min(len(lat) - 1, int(0.99 * len(lat)))], 3)},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": launches_per_frame(
                h, w, torch.cuda.get_device_properties(local).multi_processor_count) * args.steps,
            "rng_dependent_channels": int(counters.rng_dependent),
            "walk_fallback_segments": int(counters.walk_fallbacks),
            "walk_candidate_steps": int(counters.walk_candidate_steps),
            "walk_candidates": int(counters.walk_candidates),
            "walk_survivors": int(counters.walk_survivors),
        }
        if frames is not None:
            line["batched"] = run_batched(ctx, frames, args, golden)
            line["e2e_batched"] = run_e2e_batched(frames, line["batched"])
        if heavy is not None:
            line["heavy_batched"] = run_heavy(ctx, heavy, args, golden, line.get("batched"))
        if pool is not None:
            line["serving"] = run_serving(ctx, pool, args)
        if not args.no_routing:
            line["routing"] = run_routing(ctx, d_in, h, w)
        print(json.dumps(line), flush=True)


def run_routing(ctx, d_in, h, w, repeats: int = 3):
    """The at-floor routing census (hybrid routing.py:447-793) on this frame's
    own at-floor mask (score == floor), mask resident on the device.

    Times route_at_floor_mask (labelling, distance, dilation, tables, the
    three planes copied back) and serialize_routing_json on the host clock,
    and the CPU restatement of the same census (the oracle, one thread) as
    its baseline; checks the census bytes and planes against it."""

    import torch

    from fauxice_b200 import _lib, routing
    from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE
    from oracle import routing_oracle as ro

    lib = _lib.load()
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    d_out = torch.empty((h, w, 3), dtype=torch.int16, device=d_in.device)
    d_score = torch.empty((h, w), dtype=torch.float32, device=d_in.device)
    ctx.check(lib.fx_process_device(ctx.handle, d_in.data_ptr(), h, w, ctypes.byref(params), None,
                                    NIKON_PE_INITIAL_STATE, d_out.data_ptr(), d_score.data_ptr(),
                                    None, None, None))
    torch.cuda.synchronize()
    at_floor = d_score == float(DEFAULT_PROFILE.score_floor())
    routing.serialize_routing_json(routing.route_at_floor_mask(at_floor))  # warm
    census, serialize = [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        result = routing.route_at_floor_mask(at_floor)
        t1 = time.perf_counter()
        payload = routing.serialize_routing_json(result)
        census.append(t1 - t0)
        serialize.append(time.perf_counter() - t1)
    host_mask = at_floor.cpu().numpy()
    t0 = time.perf_counter()
    doc, prov, synth, final = ro.route(host_mask)
    expected = ro.serialize(doc)
    oracle_s = time.perf_counter() - t0
    exact = (payload == expected and np.array_equal(result.provisional_labels, prov)
             and np.array_equal(result.synthesis_mask, synth)
             and np.array_equal(result.final_labels, final))
    best = min(c + s for c, s in zip(census, serialize))
    return {
        "workload": f"at-floor mask of the seed-2 {h}x{w} frame ({h * w / 1e6:.1f} MP, "
                    f"{int(host_mask.sum())} at-floor pixels), default policy, device-resident",
        "regions": len(result.provisional_regions),
        "final_regions": len(result.final_regions),
        "census_ms": round(1e3 * min(census), 2),
        "serialize_ms": round(1e3 * min(serialize), 2),
        "mp_per_s": round(h * w / 1e6 / best, 1),
        "json_bytes": len(payload),
        "bit_exact_vs_oracle": bool(exact),
        "cpu_baseline": {"value": round(1e3 * oracle_s, 1), "unit": "ms", "cores": 1,
                         "kind": "port", "sample": "the same mask, census and serialization"},
        "timing": "host clock, best of 3 after one warm run",
    }


def run_batched(ctx, frames, args, golden):
    """The batched workload: 16 frames of uneven sizes, device-resident.

    Timed once with one frame in flight (the plain path on this mix) and once
    with the autotuned number of slots; every batched output is compared
    with its one-at-a-time output, and frames 0-4 (seeds 100-104) with the
    reference's recorded results.
    """

    import hashlib

    import torch

    from fauxice_b200 import batch

    d_in = [torch.from_numpy(np.ascontiguousarray(f).view(np.int16)).to("cuda") for f in frames]
    plain_out = [torch.empty((f.shape[0], f.shape[1], 3), dtype=torch.int16, device="cuda")
                 for f in frames]
    outs = [torch.empty_like(o) for o in plain_out]
    mp = sum(f.shape[0] * f.shape[1] for f in frames) / 1e6
    as_jobs = lambda dst: [batch.DeviceFrame(d.data_ptr(), f.shape[0], f.shape[1], o.data_ptr())
                           for f, d, o in zip(frames, d_in, dst)]

    def timed(jobs, slots):
        times = []
        for _ in range(args.batch_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch.run_device_batch(ctx, jobs, slots=slots)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return min(times), sorted(times)[len(times) // 2]

    import tempfile

    batch.set_walk_wave(ctx, 0)
    batch.run_device_batch(ctx, as_jobs(plain_out), slots=1)  # warm
    plain_best, plain_med = timed(as_jobs(plain_out), 1)
    with tempfile.TemporaryDirectory() as tmp:  # always measured here, never from a cache
        entry, _ = batch.autotune(ctx, as_jobs(outs), candidates=(2, 4, 8), waves=(0, 148),
                                  tiles=(8, 16), cache_path=os.path.join(tmp, "tuning.json"),
                                  retune=True)
    slots, wave, tile = entry["slots"], entry["walk_wave"], entry["stencil_tile"]
    # the tuned configuration with every launch at the default priority
    batch.set_launch_priority(ctx, False)
    unprio = [torch.empty_like(o) for o in plain_out]
    batch.run_device_batch(ctx, as_jobs(unprio), slots=slots)  # warm
    _, unprio_med = timed(as_jobs(unprio), slots)
    batch.set_launch_priority(ctx, True)
    best, med = timed(as_jobs(outs), slots)
    same = all(torch.equal(a, b) for a, b in zip(outs, plain_out))
    same = same and all(torch.equal(a, b) for a, b in zip(unprio, plain_out))
    digests = [hashlib.sha256(o.cpu().numpy().view(np.uint16).astype("<u2").tobytes()).hexdigest()
               for o in outs]
    ref_ok = [digests[i] == golden["jobs"][f"batch_{i}"]["output_sha256"] for i in range(5)]
    batch.set_walk_wave(ctx, 0)
    batch.set_stencil_tile(ctx, 0)
    return {
        "_digests": digests,
        "workload": f"{len(frames)} frames cycling 5782x3946, 3946x5782, 2892x1973, 1024x768, "
                    "4000x2700 (seeds 100-115, native defect density), device-resident",
        "value": round(mp / med, 1), "unit": "MP/s", "megapixels": round(mp, 2),
        "ms_per_step": round(1000 * med, 2), "steps": args.batch_steps,
        "plain_same_mix": {"value": round(mp / plain_med, 1), "unit": "MP/s",
                           "ms_per_step": round(1000 * plain_med, 2), "slots": 1},
        "slots": slots, "walk_wave": wave, "stencil_tile": tile,
        "launch_priority": "chain and walk at the device's greatest priority",
        "without_priority": {"value": round(mp / unprio_med, 1), "unit": "MP/s",
                             "ms_per_step": round(1000 * unprio_med, 2)},
        "tuning_ms": {f"slots={k.split(',')[0]},wave={k.split(',')[1]},tile={k.split(',')[2]}": v
                      for k, v in entry["timings_ms"].items()},
        "autotuner": "fauxice_b200.batch.autotune (slots x walk wave x stencil tile; JSON cache "
                     "keyed by device and frame shapes; remeasured for this run)",
        "timing": "host clock around the whole batch, synchronize on both sides (frames run on "
                  "several library streams)",
        "bit_exact_vs_single_frame": bool(same),
        "bit_exact_vs_reference_frames_0_4": bool(all(ref_ok)),
    }


def run_heavy(ctx, frames, args, golden, batched):
    """Config 4, heavy damage: 8 full 5782x3946 frames at ~5% coverage
    (200 floor-saturating blobs, crossing scratches; seeds 200-207),
    device-resident, one at a time and batched with the slot count the mix
    tuned; every batched output equals its single-frame output, and frames
    0-1 equal the reference's recorded results."""

    import hashlib

    import torch

    from fauxice_b200 import batch

    d_in = [torch.from_numpy(np.ascontiguousarray(f).view(np.int16)).to("cuda") for f in frames]
    plain_out = [torch.empty((f.shape[0], f.shape[1], 3), dtype=torch.int16, device="cuda")
                 for f in frames]
    outs = [torch.empty_like(o) for o in plain_out]
    mp = sum(f.shape[0] * f.shape[1] for f in frames) / 1e6
    jobs = lambda dst: [batch.DeviceFrame(d.data_ptr(), f.shape[0], f.shape[1], o.data_ptr())
                        for f, d, o in zip(frames, d_in, dst)]
    slots = batched["slots"] if batched else 4
    wave = batched["walk_wave"] if batched else 0
    tile = batched["stencil_tile"] if batched else 0

    def timed(dst, n_slots):
        times = []
        for _ in range(args.batch_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            counters = batch.run_device_batch(ctx, jobs(dst), slots=n_slots)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return sorted(times)[len(times) // 2], counters

    batch.set_walk_wave(ctx, 0)
    batch.run_device_batch(ctx, jobs(plain_out), slots=1)  # warm
    plain_med, _ = timed(plain_out, 1)
    batch.set_walk_wave(ctx, wave)
    batch.set_stencil_tile(ctx, tile)
    med, counters = timed(outs, slots)
    batch.set_walk_wave(ctx, 0)
    batch.set_stencil_tile(ctx, 0)
    same = all(torch.equal(a, b) for a, b in zip(outs, plain_out))
    ref_ok = []
    for i in range(2):
        host = outs[i].cpu().numpy().view(np.uint16)
        digest = hashlib.sha256(host.astype("<u2").tobytes()).hexdigest()
        ref_ok.append(digest == golden["jobs"][f"heavy_full_{i}"]["output_sha256"])
    return {
        "workload": f"{len(frames)} full 5782x3946 heavy-damage frames (~5% coverage incl. "
                    "200 blobs r U[20,60] with IR x U[0.01,0.1], crossing scratches; seeds "
                    "200-207), device-resident",
        "value": round(mp / med, 1), "unit": "MP/s", "megapixels": round(mp, 2),
        "ms_per_step": round(1000 * med, 2), "steps": args.batch_steps,
        "plain_same_mix": {"value": round(mp / plain_med, 1), "unit": "MP/s",
                           "ms_per_step": round(1000 * plain_med, 2), "slots": 1},
        "slots": slots, "walk_wave": wave, "stencil_tile": tile or 8,
        "attempted_pixels": int(sum(c.attempted for c in counters)),
        "rng_dependent_channels": int(sum(c.rng_dependent for c in counters)),
        "capacity_reruns": int(sum(c.capacity_reruns for c in counters)),
        "timing": "host clock around the whole batch, synchronize on both sides",
        "bit_exact_vs_single_frame": bool(same),
        "bit_exact_vs_reference_frames_0_1": bool(all(ref_ok)),
    }


def run_e2e_batched(frames, batched):
    """The batched mix through the public host-buffer API: 16 jobs of host
    numpy frames into process_batch (validation, prepass, staged uploads,
    passes, downloads and output SHA-256 digests all inside the timed
    region), with the slot count the device-resident run tuned."""

    from fauxice_b200 import batch, synthetic

    digests = batched.pop("_digests")
    jobs = [make_job(f, synthetic.make_prepass(f)) for f in frames]
    batch.process_batch(jobs, slots=batched["slots"])  # warm: pinned staging of every slot
    t0 = time.perf_counter()
    results = batch.process_batch(jobs, slots=batched["slots"])
    elapsed = time.perf_counter() - t0
    mp = sum(f.shape[0] * f.shape[1] for f in frames) / 1e6
    exact = all(r.replay.output_sha256 == d for r, d in zip(results, digests))
    return {"value": round(mp / elapsed, 1), "unit": "MP/s", "ms_per_step": round(1e3 * elapsed, 1),
            "frames": len(frames), "slots": batched["slots"],
            "h2d_bytes_per_step": int(sum(f.nbytes for f in frames)),
            "d2h_bytes_per_step": int(sum(f.shape[0] * f.shape[1] * 6 for f in frames)),
            "bit_exact_vs_device_batch": bool(exact),
            "api": "fauxice_b200.batch.process_batch(jobs) (host numpy in/out, output SHA-256 "
                   "per frame on a thread pool)"}


def run_serving(ctx, pool, args):
    """Requests at Poisson rates over a shortened window; sizes 50% 5782x3946,
    30% 2892x1973, 20% crops of U[256, 2048]^2, each pool frame with its own
    defect coverage from U[0.1%, 3%]; inputs in pinned host memory.

    Admission by device memory, latency from arrival to the output in host
    memory, every output compared on the device with the same frame's
    single-frame output."""

    import torch

    from fauxice_b200 import _lib, serve
    from fauxice_b200.profile import DEFAULT_PROFILE, NIKON_PE_INITIAL_STATE

    lib = _lib.load()
    params = DEFAULT_PROFILE.hot_path_parameters().to_c()
    frames, specs = pool
    pinned, expected = [], []
    for f in frames:
        h, w = f.shape[:2]
        pinned.append(torch.from_numpy(np.ascontiguousarray(f).view(np.int16)).pin_memory())
        d_in = pinned[-1].to("cuda")
        out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
        torch.cuda.synchronize()
        # synchronous (counters given): d_in may be reused once this returns
        ctx.check(lib.fx_process_device(ctx.handle, d_in.data_ptr(), h, w, ctypes.byref(params),
                                        None, NIKON_PE_INITIAL_STATE, out.data_ptr(), None, None,
                                        None, ctypes.byref(_lib.FxCounters())))
        expected.append(out)
    torch.cuda.synchronize()
    groups = [[k for k, s in enumerate(specs) if (s[1], s[2]) == (5782, 3946)],
              [k for k, s in enumerate(specs) if (s[1], s[2]) == (2892, 1973)],
              [k for k, s in enumerate(specs) if (s[1], s[2]) not in ((5782, 3946), (2892, 1973))]]
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    out = {"workload": "Poisson arrivals, 50% 5782x3946 / 30% 2892x1973 / 20% crops "
                       "U[256,2048]^2, per-frame defect coverage U[0.1%,3%] (pool of 16 "
                       f"frames), {args.serve_seconds:g} s per rate (of the 120 s workload); "
                       "admission by free HBM (fx_frame_bytes), up to 12 in flight; latency "
                       "from arrival to the RGB16 output in pinned host memory; every output "
                       "compared on the device with its frame's single-frame output",
           "pool_coverage": [round(s[3], 4) for s in specs], "rates": {}}
    for r_i, rate in enumerate(rates):
        arrivals = serve.poisson_arrivals(rate, args.serve_seconds, seed=600 + r_i)
        pick = np.random.default_rng(700 + r_i)
        requests = []
        for t in arrivals:
            u = pick.random()
            group = groups[0] if u < 0.5 else (groups[1] if u < 0.8 else groups[2])
            k = group[int(pick.integers(0, len(group)))]
            requests.append(serve.Request(float(t), pinned[k], expected[k]))
        report = serve.serve(ctx, requests, max_slots=12)
        out["rates"][f"{rate:g}/s"] = report.summary()
    return out


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch under torch.distributed.run
        sys.exit(subprocess.call(launch_command(args.gpus, sys.argv[1:], free_port())))
    world, rank, local = dist_setup(args.plan_only)
    if args.plan_only:
        run_plan(world, rank)
    elif args.impl == "reference":
        run_reference(args, world, rank)
    elif args.impl == "numba":
        run_numba(args, world, rank)
    elif args.serve_only:
        if rank == 0:
            from fauxice_b200 import engine

            specs = serving_pool_specs()
            pool = (generate(_serving_frame, specs), specs)
            import torch

            torch.cuda.set_device(local)
            report = run_serving(engine.context(local), pool, args)
            print(json.dumps({"metric": METRIC, "serving": report}), flush=True)
    else:
        frames = heavy = pool = None
        if world == 1 and not args.no_batch:
            frames = generate(_batch_frame, list(range(BATCH_FRAMES)))
            if not args.no_heavy:
                heavy = generate(_heavy_frame, list(range(HEAVY_FRAMES)))
            specs = serving_pool_specs()
            pool = (generate(_serving_frame, specs), specs)
        run_b200(args, world, rank, local, frames, heavy, pool)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
