"""Seeded input recipes for the golden parity cases.

Each recipe restates how the reference's own tests build an input (cited by
file:line, paths relative to the reference repository) but with a fixed
seed, so the inputs are identical in every process.  ``make_golden.py`` runs
the reference on these inputs (in a container where the reference is
importable) and records the results in ``reference_results.json``; the tests
rebuild the same inputs from these recipes and compare.
"""

from __future__ import annotations

import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
_PKG = os.path.join(_ROOT, "digital-fauxice_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from fauxice_b200 import synthetic  # noqa: E402


def conftest_rgbi(height: int, width: int, *, offset: int) -> np.ndarray:
    """tests/conftest.py:16-25 (synthetic_rgbi)."""

    y, x = np.indices((height, width), dtype=np.uint32)
    pixels = np.empty((height, width, 4), dtype=np.uint16)
    pixels[:, :, 0] = (12_000 + offset + 53 * y + 97 * x).astype(np.uint16)
    pixels[:, :, 1] = (16_000 + offset + 67 * y + 71 * x).astype(np.uint16)
    pixels[:, :, 2] = (20_000 + offset + 89 * y + 43 * x).astype(np.uint16)
    pixels[:, :, 3] = (44_000 + offset + 31 * y + 29 * x).astype(np.uint16)
    return pixels


def engine_8x8():
    """tests/conftest.py:28-53: the 8x8 job pinned by tests/test_engine.py:28-33."""

    main = conftest_rgbi(8, 8, offset=150)
    main[3:5, 3:5, 3] = np.uint16(9_000)
    return main, conftest_rgbi(8, 8, offset=0)


def hybrid_256():
    """hybrid/examples/make_synthetic_inputs.py:21-46 (the 256x256 example)."""

    def frame(offset: int) -> np.ndarray:
        y, x = np.indices((256, 256), dtype=np.uint32)
        f = np.empty((256, 256, 4), dtype=np.uint16)
        f[:, :, 0] = (12_000 + offset + 31 * y + 47 * x).astype(np.uint16)
        f[:, :, 1] = (16_000 + offset + 43 * y + 29 * x).astype(np.uint16)
        f[:, :, 2] = (20_000 + offset + 37 * y + 41 * x).astype(np.uint16)
        f[:, :, 3] = (45_000 + offset + 17 * y + 13 * x).astype(np.uint16)
        return f

    main = frame(120)
    main[110:130, 118:138, 3] = np.uint16(0)
    return main, frame(0)


def self_test_job():
    """src/portable_digital_ice/backend.py:60-87 (_synthetic_self_test_job)."""

    rng = np.random.default_rng(20260716)
    height, width = 48, 64
    main = rng.integers(20000, 60000, size=(height, width, 4), dtype=np.uint16)
    main[18:26, 30:39, 3] = rng.integers(200, 2000, size=(8, 9), dtype=np.uint16)
    main[0:2, 0:6, 3] = 500
    main[-2:, -6:, 3] = 700
    main[3, width - 3, 3] = 900
    prepass = rng.integers(20000, 60000, size=(24, 32, 4), dtype=np.uint16)
    prepass[10:14, 12:17, 3] = 300
    return main, prepass


TILE_CASES = (
    "uniform",
    "impulse",
    "edge",
    "checkerboard",
    "high_dynamic_range",
    "corner_dust",
    "edge_band_dust",
    "epoch_boundary_dust",
    "threshold_straddle",
    "final_block_six_rows",
)


def adversarial_tile(case: str):
    """tests/test_fast_cpu_differential.py:100-176 with seed 7000+index
    (the reference seeds with abs(hash(case)), which varies per process)."""

    rng = np.random.default_rng(7000 + TILE_CASES.index(case))
    height, width = 41, 64
    if case == "final_block_six_rows":
        height = 30
    main = rng.integers(18000, 62000, size=(height, width, 4), dtype=np.uint16)
    if case == "uniform":
        main[:] = 43210
        main[:, :, 3] = 51234
    elif case == "impulse":
        main[:] = 40000
        main[height // 2, width // 2] = (65535, 0, 65535, 60000)
        main[height // 2, width // 2 + 1, 3] = 100
    elif case == "edge":
        main[:, : width // 2] = (15000, 16000, 17000, 52000)
        main[:, width // 2 :] = (60000, 59000, 58000, 52000)
        main[:, width // 2 - 1 : width // 2 + 1, 3] = 800
    elif case == "checkerboard":
        yy, xx = np.mgrid[0:height, 0:width]
        board = ((yy + xx) % 2).astype(np.uint16)
        for c in range(3):
            main[:, :, c] = 20000 + board * 30000
        main[:, :, 3] = 50000 + board * 10000
    elif case == "high_dynamic_range":
        main[:, :, :3] = rng.choice(
            np.array([0, 1, 2, 32768, 65533, 65534, 65535], dtype=np.uint16),
            size=(height, width, 3),
        )
        main[:, :, 3] = rng.choice(
            np.array([0, 8847, 8848, 8849, 65535], dtype=np.uint16), size=(height, width)
        )
    elif case == "corner_dust":
        for (y0, x0) in ((0, 0), (0, width - 3), (height - 3, 0), (height - 3, width - 3)):
            main[y0 : y0 + 3, x0 : x0 + 3, 3] = 500
    elif case == "edge_band_dust":
        main[0:4, :, 3] = rng.integers(100, 3000, size=(4, width), dtype=np.uint16)
        main[:, 0:4, 3] = rng.integers(100, 3000, size=(height, 4), dtype=np.uint16)
        main[:, width - 4 :, 3] = rng.integers(100, 3000, size=(height, 4), dtype=np.uint16)
        main[height - 4 :, :, 3] = rng.integers(100, 3000, size=(4, width), dtype=np.uint16)
    elif case == "epoch_boundary_dust":
        main[7:9, :, 3] = 600
        main[15:17, 24:40, 3] = 700
        main[23:25, :, 3] = rng.integers(100, 9000, size=(2, width), dtype=np.uint16)
    elif case == "threshold_straddle":
        main[:, :, 3] = rng.choice(
            np.array([8846, 8847, 8848, 8849, 8850], dtype=np.uint16), size=(height, width)
        )
    elif case == "final_block_six_rows":
        main[height - 6 :, :, 3] = rng.integers(100, 4000, size=(6, width), dtype=np.uint16)
    prepass = rng.integers(15000, 62000, size=(24, 32, 4), dtype=np.uint16)
    prepass[6:10, 8:13, 3] = 400
    return main, prepass


def diagnostics_30x40():
    """tests/test_fast_cpu_differential.py:397-407."""

    rng = np.random.default_rng(20260722)
    main = rng.integers(18000, 62000, size=(30, 40, 4), dtype=np.uint16)
    main[8:14, 12:22, 3] = 550
    main[0:2, 0:6, 3] = 500
    main[-2:, -6:, 3] = 700
    prepass = rng.integers(15000, 62000, size=(24, 32, 4), dtype=np.uint16)
    prepass[6:10, 8:13, 3] = 400
    return main, prepass


def multi_band_300x16():
    """tests/test_fast_cpu_differential.py:410-427."""

    rng = np.random.default_rng(20260725)
    height, width = 300, 16
    main = rng.integers(18000, 62000, size=(height, width, 4), dtype=np.uint16)
    main[120:136, 4:12, 3] = rng.integers(200, 2500, size=(16, 8), dtype=np.uint16)
    main[250:262, 2:10, 3] = rng.integers(200, 2500, size=(12, 8), dtype=np.uint16)
    main[290:298, 6:14, 3] = 700
    sy = rng.integers(0, height, size=150)
    sx = rng.integers(0, width, size=150)
    main[sy, sx, 3] = rng.integers(200, 3000, size=150).astype(np.uint16)
    prepass = rng.integers(15000, 62000, size=(24, 32, 4), dtype=np.uint16)
    prepass[6:10, 8:13, 3] = 400
    return main, prepass


def generated(seed: int, height: int, width: int, spec: str = "native"):
    """A frame from the benchmark generator at an arbitrary size."""

    base = {"native": synthetic.NATIVE_FRAME, "small": synthetic.SMALL_CROP,
            "heavy": synthetic.HEAVY_FRAME}[spec]
    main = synthetic.make_frame(seed, height, width,
                                synthetic.scaled_spec(base, height, width))
    return main, synthetic.make_prepass(main)


def native_crop(index: int, size: int = 256):
    """Crop i of the seed-2 native frame at origin default_rng(1000+i); the
    crop reuses the parent frame's prepass."""

    main, prepass = synthetic.native_frame(2)
    (y0, x0), = synthetic.crop_origins(main.shape[0], main.shape[1], size, 1, 1000 + index)
    return np.ascontiguousarray(main[y0 : y0 + size, x0 : x0 + size]), prepass


# Jobs checked against process_cpu (pure Python) or, for large frames,
# against the reference's cpu-fast backend.
JOB_CASES = {
    "engine_8x8": (engine_8x8, "cpu"),
    "hybrid_256": (hybrid_256, "cpu"),
    "self_test_48x64": (self_test_job, "cpu"),
    "diagnostics_30x40": (diagnostics_30x40, "cpu"),
    "multi_band_300x16": (multi_band_300x16, "cpu"),
    **{f"tile_{c}": ((lambda c=c: adversarial_tile(c)), "cpu") for c in TILE_CASES},
    **{f"gen_{s}_{h}x{w}": ((lambda s=s, h=h, w=w: generated(s, h, w)), "cpu")
       for s, h, w in ((3, 37, 45), (4, 64, 64), (5, 96, 80), (6, 130, 70), (7, 5, 8),
                       (8, 6, 9), (9, 17, 200))},
    "small_crop_512": ((lambda: synthetic.small_crop(1)), "cpu"),
    **{f"native_crop_{i}": ((lambda i=i: native_crop(i)), "cpu") for i in range(10)},
    "heavy_1024": ((lambda: generated(201, 1024, 1024, "heavy")), "cpu-fast"),
    "native_full": ((lambda: synthetic.native_frame(2)), "cpu-fast"),
    **{f"batch_{i}": ((lambda i=i: synthetic.batch_frame(i)), "cpu-fast") for i in range(5)},
    # heavy-damage full frames (about 5% coverage, 200 floor-saturating blobs)
    **{f"heavy_full_{i}": ((lambda i=i: synthetic.heavy_full_frame(i)), "cpu-fast")
       for i in range(2)},
}

# Streaming-replay cases with explicit parameters
# (tests/test_fast_cpu_differential.py:188-395).
DIRECT_BASE = {
    "aux": {"alpha": 0.32, "offset": 1.0, "replacement": None},
    "score": {"base": 52215.4, "addend": -119.40625, "scale": -0.0010412337, "offset": 1.0,
              "floor": 0.02, "cutoff": 550},
    "decision": {"threshold": 49383.234, "count_limit": 8, "radius": 1},
    "recon": {
        "metric": 500, "cutoff": 1600, "coarse_enabled": True, "coarse": 52215.4,
        "slopes": [1.1, 1.1, 1.1], "band_enabled": [True, True, True],
        "band_scales": [1.25, 1.25, 1.25],
        "factors_a": [[1.21, 1.23, 1.13], [1.17, 1.14, 1.08], [1.04, 0.93, 0.97]],
        "factors_b": [[1.09, 1.13, 1.04], [1.08, 1.05, 1.02], [0.96, 0.84, 0.89]],
        "strengths": [0.0, 0.0, 0.0], "gate_primary": True, "gate_secondary": True,
        "row_gate": 0, "dither_scales": [0.015, 0.015, 0.025],
    },
}


def _direct_pixels(seed, h, w, box, ir):
    rng = np.random.default_rng(seed)
    px = rng.integers(15000, 64000, size=(h, w, 4), dtype=np.uint16)
    if box is not None:
        (y0, y1, x0, x1) = box
        px[y0:y1, x0:x1, 3] = ir
    return px


DIRECT_CASES = {
    # name: (seed, h, w, dust box, dust IR, parameter overrides)
    "center_only_500": (500500, 26, 48, (9, 14, 20, 29), 700, {}),
    "cross_neighbor_4000": (500501, 26, 48, (9, 14, 20, 29), 700,
                            {"recon": {"metric": 4000}}),
    "gates_off": (99, 17, 40, (5, 9, 10, 19), 900,
                  {"recon": {"metric": 4000, "gate_primary": False, "gate_secondary": False}}),
    "row_gate_3": (99, 17, 40, (5, 9, 10, 19), 900, {"recon": {"metric": 4000, "row_gate": 3}}),
    "min_height_center_only": (4004, 4, 12, (1, 3, 4, 8), 600, {"recon": {"metric": 500}}),
    "min_geometry_cross": (4005, 5, 8, (1, 3, 2, 6), 600, {"recon": {"metric": 4000}}),
    "width_one_center_only": (1001, 6, 1, (2, 4, 0, 1), 500, {"recon": {"metric": 500}}),
    "all_fallback": (2002, 10, 20, (0, 10, 0, 20), 500, {"recon": {"metric": 4000}}),
    "row_gate_7": (3003, 12, 24, (4, 8, 8, 16), 500, {"recon": {"metric": 4000, "row_gate": 7}}),
    "alpha_one": (7007, 14, 24, (5, 9, 10, 18), 650,
                  {"recon": {"metric": 4000},
                   "aux": {"alpha": 1.0, "replacement": 41234.5}}),
    "radius4_hmin": (4242, 33, 57, (10, 20, 15, 40), 800,
                     {"recon": {"metric": 4000}, "decision": {"radius": 4},
                      "score": {"cutoff": 550}}),
    "strengths_set": (4343, 29, 41, (8, 15, 12, 25), 750,
                      {"recon": {"metric": 4000, "strengths": [0.5, 0.25, 0.75],
                                 "band_enabled": [True, False, True]}}),
}


def direct_case(name: str):
    seed, h, w, box, ir, overrides = DIRECT_CASES[name]
    spec = {k: dict(v) for k, v in DIRECT_BASE.items()}
    for group, values in overrides.items():
        spec[group].update(values)
    # score.resolution_metric follows the reconstruction metric
    spec["score"]["metric"] = spec["recon"]["metric"]
    return _direct_pixels(seed, h, w, box, ir), spec


# Producer geometries (tests/test_fast_cpu_producer_parity.py:60-126).
PRODUCER_CASES = (
    (48, 64, 20260716),
    (41, 64, 11),
    (30, 40, 22),
    (8, 8, 33),
    (7, 16, 44),
    (9, 17, 55),
    (12, 24, 66),
    (25, 33, 77),
)


def producer_pixels(height: int, width: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pixels = rng.integers(0, 65536, size=(height, width, 4), dtype=np.uint16)
    straddle = rng.random(size=(height, width)) < 0.25
    pixels[:, :, 3][straddle] = rng.choice(
        np.array([8846, 8847, 8848, 8849], dtype=np.uint16), size=int(straddle.sum())
    )
    pixels[height // 3 : height // 3 + 3, : min(width, 12), 3] = 500
    return pixels
