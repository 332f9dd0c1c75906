#!/usr/bin/env python3
"""Generate tests/golden/reference_results.json by running the reference.

This script imports the reference package portable_digital_ice from
``--reference`` (or the FAUXICE_REFERENCE_SRC environment variable: the
reference checkout's ``src`` directory) and records, for every case in
cases.py, the reference's output digest, replay counters, startup receipt,
diagnostics digests and prelude records.  It is run once, in a container
where the reference is importable; the tests then need only the JSON file.

Usage: python tests/golden/make_golden.py [--only REGEX] [--skip-slow]
"""

from __future__ import annotations

import argparse
import functools
import hashlib
import json
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_results.json")


def sha(array: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("FAUXICE_REFERENCE_SRC"),
                        help="the reference checkout's src directory")
    parser.add_argument("--only", default=None)
    parser.add_argument("--skip-slow", action="store_true")
    args = parser.parse_args()
    if not args.reference:
        parser.error("give --reference or set FAUXICE_REFERENCE_SRC")
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/fauxice_numba_cache")
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, args.reference)
    sys.path.insert(0, HERE)

    import cases  # noqa: E402
    from fauxice_b200 import synthetic  # noqa: E402
    from portable_digital_ice import (  # noqa: E402
        AcquisitionEpoch, DualRGBIAcquisition, ProcessingJob, ProcessingMode, RGBI16Frame,
        ScannerModel, process_cpu,
    )
    from portable_digital_ice.dither import DitherBounds  # noqa: E402
    from portable_digital_ice.prepass import reduce_prepass_frame  # noqa: E402
    from portable_digital_ice.producer_parameters import (  # noqa: E402
        derive_producer_record_schedule,
    )
    from portable_digital_ice.profile import DEFAULT_PROFILE  # noqa: E402
    from portable_digital_ice.reconstruction import ReconstructionParameters  # noqa: E402
    from portable_digital_ice.rng import LCG24  # noqa: E402
    from portable_digital_ice.streaming import run_streaming_replay  # noqa: E402
    from portable_digital_ice.x3a import (  # noqa: E402
        AuxiliaryParameters, DecisionParameters, ScoreParameters, SharedLookupInputResponse,
    )

    # The seed-2 native frame is the parent of ten crops; build it once.
    synthetic.native_frame = functools.lru_cache(maxsize=2)(synthetic.native_frame)

    results = {}
    if os.path.exists(OUT):
        with open(OUT) as handle:
            results = json.load(handle)
    results.setdefault("jobs", {})
    results.setdefault("direct", {})
    results.setdefault("producer", {})
    response = SharedLookupInputResponse.nikon_logarithmic()

    def job(main, prepass, fid):
        return ProcessingJob(
            acquisition=DualRGBIAcquisition(
                prepass=RGBI16Frame(prepass, AcquisitionEpoch.PREPASS, 285, fid + "-pp"),
                main=RGBI16Frame(main, AcquisitionEpoch.MAIN, 4000, fid + "-main"),
                same_frame_id=fid,
            ),
            scanner_model=ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED,
            mode=ProcessingMode.NORMAL,
            selector=8,
            resolution_metric=4000,
            bit_depth=16,
            focus_exposure_locked=True,
        )

    def wanted(name):
        return args.only is None or re.search(args.only, name)

    for name, (recipe, backend) in cases.JOB_CASES.items():
        if not wanted(name):
            continue
        if args.skip_slow and (backend == "cpu-fast" or name.startswith(("small_crop", "native_crop"))):
            continue
        main, prepass = recipe()
        t0 = time.time()
        if backend == "cpu":
            res = process_cpu(job(main, prepass, name), export_diagnostics=True)
        else:
            from portable_digital_ice.fast_cpu import process_cpu_fast

            res = process_cpu_fast(job(main, prepass, name), export_diagnostics=True)
        elapsed = time.time() - t0
        reduction = reduce_prepass_frame(
            RGBI16Frame(prepass, AcquisitionEpoch.PREPASS, 285, "pp"),
            parameters=DEFAULT_PROFILE.prepass_parameters(), frame_index=0,
            evidence_id="pp", response=response,
        )
        schedule = derive_producer_record_schedule(main, response.table)
        rep = res.replay
        results["jobs"][name] = {
            "backend": backend,
            "shape": list(main.shape),
            "input_sha256": sha(main.astype("<u2")),
            "output_sha256": rep.output_sha256,
            "attempted_pixels": rep.attempted_pixels,
            "written_pixels": rep.written_pixels,
            "public_rng_advances": rep.public_rng_advances,
            "final_rng_state": rep.final_rng_state,
            "changed_pixels": rep.changed_pixels,
            "startup_attempted": list(rep.startup.attempted_per_stage),
            "startup_advances": list(rep.startup.rng_advances_per_stage),
            "startup_final_state": rep.startup.final_rng_state,
            "score_plane_sha256": sha(res.diagnostics.score_plane.astype("<f4")),
            "at_floor_sha256": sha(res.diagnostics.at_floor_mask),
            "changed_mask_sha256": sha(res.diagnostics.changed_mask),
            "prepass_payload": reduction.record.payload.hex(),
            "prepass_valid_pixels": reduction.valid_pixels,
            "prepass_fully_valid_tiles": reduction.fully_valid_tiles,
            "producer_payloads_sha256": hashlib.sha256(b"".join(schedule.record_payloads)).hexdigest(),
            "reference_seconds": round(elapsed, 3),
        }
        print(f"{name}: {backend} {elapsed:.1f}s attempted={rep.attempted_pixels}", flush=True)
        with open(OUT, "w") as handle:
            json.dump(results, handle, indent=1, sort_keys=True)

    for name in cases.DIRECT_CASES:
        if not wanted(name):
            continue
        pixels, spec = cases.direct_case(name)
        a, s, d, r = spec["aux"], spec["score"], spec["decision"], spec["recon"]
        aux = AuxiliaryParameters(selected_visible_channel=0, alpha=float(np.float32(a["alpha"])),
                                  calibration_offset=a["offset"],
                                  alpha_one_replacement=(None if a["replacement"] is None
                                                         else float(np.float32(a["replacement"]))))
        score = ScoreParameters(base_primary=float(np.float32(s["base"])),
                                base_addend=float(np.float32(s["addend"])),
                                scale=float(np.float32(s["scale"])), offset=s["offset"],
                                floor=float(np.float32(s["floor"])), resolution_metric=s["metric"],
                                horizontal_minimum_resolution_cutoff=s["cutoff"])
        decision = DecisionParameters(sample_threshold=float(np.float32(d["threshold"])),
                                      count_limit=d["count_limit"], perpendicular_radius=d["radius"])
        recon = ReconstructionParameters(
            resolution_metric=r["metric"], cross_neighbor_cutoff=r["cutoff"],
            coarse_enabled=r["coarse_enabled"], coarse_reference=float(np.float32(r["coarse"])),
            coarse_slopes=tuple(r["slopes"]), band_enabled=tuple(r["band_enabled"]),
            band_scales=tuple(r["band_scales"]),
            factors_a=tuple(tuple(v) for v in r["factors_a"]),
            factors_b=tuple(tuple(v) for v in r["factors_b"]),
            configured_strengths=tuple(r["strengths"]), driver_gate_primary=r["gate_primary"],
            driver_gate_secondary=r["gate_secondary"], row_reconstruction_gate=r["row_gate"],
            dither_scales=tuple(r["dither_scales"]),
        )
        bounds = DitherBounds.from_lookup(response.table, maximum_index=65535)
        out = np.empty((pixels.shape[0], pixels.shape[1], 3), np.uint16)
        rep = run_streaming_replay(pixels, out, response=response, auxiliary_parameters=aux,
                                   score_parameters=score, decision_parameters=decision,
                                   reconstruction_parameters=recon, dither_bounds=bounds,
                                   generator=LCG24.from_nikon_pe_initial_state())
        results["direct"][name] = {
            "output_sha256": rep.output_sha256,
            "attempted_pixels": rep.attempted_pixels,
            "written_pixels": rep.written_pixels,
            "public_rng_advances": rep.public_rng_advances,
            "final_rng_state": rep.final_rng_state,
            "changed_pixels": rep.changed_pixels,
            "startup_attempted": list(rep.startup.attempted_per_stage),
            "startup_advances": list(rep.startup.rng_advances_per_stage),
            "startup_final_state": rep.startup.final_rng_state,
        }
        print(f"direct {name}: attempted={rep.attempted_pixels}", flush=True)

    for h, w, seed in cases.PRODUCER_CASES:
        name = f"{h}x{w}_seed{seed}"
        if not wanted(name):
            continue
        pixels = cases.producer_pixels(h, w, seed)
        schedule = derive_producer_record_schedule(pixels, response.table)
        results["producer"][name] = {
            "payloads_sha256": hashlib.sha256(b"".join(schedule.record_payloads)).hexdigest(),
            "input_scale_sha256": sha(schedule.input_scale.astype("<f4")),
            "scaled_input_sha256": sha(schedule.scaled_input.astype("<f4")),
            "mean_visible_sha256": sha(
                schedule.mean_schedule.calibration_mean_visible.astype("<f4")),
            "mean_infrared_sha256": sha(
                schedule.mean_schedule.calibration_mean_infrared.astype("<f4")),
        }
    with open(OUT, "w") as handle:
        json.dump(results, handle, indent=1, sort_keys=True)
    print("wrote", OUT)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
