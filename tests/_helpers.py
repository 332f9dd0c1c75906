"""Shared test helpers: jobs, digests and golden comparisons."""

from __future__ import annotations

import hashlib
import time

import numpy as np

import cases
from fauxice_b200 import contracts
from fauxice_b200 import streaming as b200_streaming

# Golden job cases cheap enough for the CPU oracle in the default suite.
SLOW_JOBS = {"native_full", "batch_0", "batch_1", "batch_2", "batch_3", "batch_4",
             "heavy_full_0", "heavy_full_1"}


def sha(array: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def make_job(main: np.ndarray, prepass: np.ndarray, frame_id: str = "test"):
    acquisition = contracts.DualRGBIAcquisition(
        prepass=contracts.RGBI16Frame(prepass, contracts.AcquisitionEpoch.PREPASS, 285,
                                      frame_id + "-pp"),
        main=contracts.RGBI16Frame(main, contracts.AcquisitionEpoch.MAIN, 4000,
                                   frame_id + "-main"),
        same_frame_id=frame_id,
    )
    return contracts.ProcessingJob(
        acquisition=acquisition,
        scanner_model=contracts.ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED,
        mode=contracts.ProcessingMode.NORMAL,
        selector=8,
        resolution_metric=4000,
        bit_depth=16,
        focus_exposure_locked=True,
    )


def job_mismatches(expected: dict, *, output_sha256, attempted, written, advances, final_state,
                   changed, startup_attempted, startup_advances, startup_final_state,
                   score=None, at_floor=None, changed_mask=None) -> list[str]:
    got = {
        "output_sha256": output_sha256,
        "attempted_pixels": attempted,
        "written_pixels": written,
        "public_rng_advances": advances,
        "final_rng_state": final_state,
        "changed_pixels": changed,
        "startup_attempted": list(startup_attempted),
        "startup_advances": list(startup_advances),
        "startup_final_state": startup_final_state,
    }
    bad = [f"{k}: expected {expected[k]} got {v}" for k, v in got.items() if expected[k] != v]
    if score is not None and "score_plane_sha256" in expected:
        if sha(score.astype("<f4")) != expected["score_plane_sha256"]:
            bad.append("score plane")
        if sha(at_floor) != expected["at_floor_sha256"]:
            bad.append("at-floor mask")
        if sha(changed_mask) != expected["changed_mask_sha256"]:
            bad.append("changed mask")
    return bad


def oracle_mismatches(expected: dict, res) -> list[str]:
    return job_mismatches(
        expected, output_sha256=res.output_sha256, attempted=res.attempted_pixels,
        written=res.written_pixels, advances=res.public_rng_advances,
        final_state=res.final_rng_state, changed=res.changed_pixels,
        startup_attempted=res.startup_attempted, startup_advances=res.startup_advances,
        startup_final_state=res.startup_final_state, score=res.score_plane,
        at_floor=res.at_floor_mask, changed_mask=res.changed_mask)


def b200_mismatches(expected: dict, result) -> list[str]:
    rep = result.replay
    diag = result.diagnostics
    return job_mismatches(
        expected, output_sha256=rep.output_sha256, attempted=rep.attempted_pixels,
        written=rep.written_pixels, advances=rep.public_rng_advances,
        final_state=rep.final_rng_state, changed=rep.changed_pixels,
        startup_attempted=rep.startup.attempted_per_stage,
        startup_advances=rep.startup.rng_advances_per_stage,
        startup_final_state=rep.startup.final_rng_state,
        score=diag.score_plane if diag else None, at_floor=diag.at_floor_mask if diag else None,
        changed_mask=diag.changed_mask if diag else None)


def direct_objects(spec: dict):
    """Reference-style parameter objects for a direct replay case."""

    a, s, d, r = spec["aux"], spec["score"], spec["decision"], spec["recon"]
    f = lambda v: float(np.float32(v))  # noqa: E731
    aux = b200_streaming.AuxiliaryParameters(
        0, f(a["alpha"]), a["offset"], None if a["replacement"] is None else f(a["replacement"]))
    score = b200_streaming.ScoreParameters(f(s["base"]), f(s["addend"]), f(s["scale"]),
                                           s["offset"], f(s["floor"]), s["metric"], s["cutoff"])
    decision = b200_streaming.DecisionParameters(f(d["threshold"]), d["count_limit"], d["radius"])
    recon = b200_streaming.ReconstructionParameters(
        r["metric"], r["cutoff"], r["coarse_enabled"], f(r["coarse"]), tuple(r["slopes"]),
        tuple(r["band_enabled"]), tuple(r["band_scales"]),
        tuple(tuple(v) for v in r["factors_a"]), tuple(tuple(v) for v in r["factors_b"]),
        tuple(r["strengths"]), r["gate_primary"], r["gate_secondary"], r["row_gate"],
        tuple(r["dither_scales"]))
    return aux, score, decision, recon


def oracle_direct(pixels: np.ndarray, spec: dict):
    """Run a direct case on the oracle (parameters quantised as the reference does)."""

    from oracle import oracle as ox

    aux, score, decision, recon = direct_objects(spec)
    params = ox.Params(
        score_addend=score.base_addend, score_scale=score.scale, score_offset=score.offset,
        score_floor=score.floor,
        horizontal_minimum=score.horizontal_minimum_resolution_cutoff < score.resolution_metric,
        visible_channel=0, decision_threshold=decision.sample_threshold,
        count_limit=decision.count_limit, radius=decision.perpendicular_radius,
        cross_neighbor=recon.resolution_metric > recon.cross_neighbor_cutoff,
        coarse_enabled=recon.coarse_enabled, coarse_slopes=recon.coarse_slopes,
        band_enabled=recon.band_enabled, band_scales=recon.band_scales,
        factors_a=tuple(v for row in recon.factors_a for v in row),
        factors_b=tuple(v for row in recon.factors_b for v in row),
        configured_strengths=recon.configured_strengths,
        driver_gate_primary=recon.driver_gate_primary, dither_scales=recon.dither_scales)
    stages = ox.constant_stage_table(
        pixels.shape[0], alpha=aux.alpha, offset=aux.calibration_offset,
        replacement=aux.alpha_one_replacement, score_base=score.base_primary,
        coarse=recon.coarse_reference, gate_secondary=recon.driver_gate_secondary,
        row_gate=recon.row_reconstruction_gate)
    return ox.replay(pixels, stages, params, diagnostics=False)


class Timer:
    def __enter__(self):
        self.t = time.perf_counter()
        return self

    def __exit__(self, *exc):
        self.elapsed = time.perf_counter() - self.t
