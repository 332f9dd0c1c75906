"""Seeded synthetic RGBI scans standing in for the reference's private frames.

The reference validates on two private 4000 dpi scans that are not shipped.
These generators produce film-scan-like uint16 RGBI frames with the shapes and
value distributions of the benchmark workloads:

* RGB: 30000 plus three seeded low-frequency 2-D sinusoids per channel
  (0.5-3 cycles per frame, total amplitude about 12000) plus Gaussian grain
  (sigma 600), clipped to 0..65535.
* IR: 52000 plus Gaussian noise (sigma 400).
* Defects: dark discs and polyline scratches (width 1-3 px).  Each defect
  multiplies IR by U[ir_lo, ir_hi] and RGB by U[0.3, 0.9].
* Prepass: a deterministic stride-14 decimation of the defected main frame
  (4000 dpi / 285 dpi is about 14.04).

Everything is a pure function of the seed.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FULL_FRAME = (5782, 3946)
PREPASS_STRIDE = 14


@dataclass(frozen=True)
class DefectSpec:
    discs: int
    disc_radius: tuple[float, float]
    scratches: int
    scratch_length: tuple[float, float]
    ir_factor: tuple[float, float] = (0.05, 0.7)
    rgb_factor: tuple[float, float] = (0.3, 0.9)
    blobs: int = 0
    blob_radius: tuple[float, float] = (20.0, 60.0)
    blob_ir_factor: tuple[float, float] = (0.01, 0.1)


# Small crop (512x512): 40 discs r~U[2,12], 6 scratches.
SMALL_CROP = DefectSpec(discs=40, disc_radius=(2, 12), scratches=6, scratch_length=(30, 400))
# Native frame: ~3000 discs r~U[1,20], 60 scratches of length U[50,2000] (~0.5%).
NATIVE_FRAME = DefectSpec(discs=3000, disc_radius=(1, 20), scratches=60,
                          scratch_length=(50, 2000))
# Dense damage for small stress frames: about 27% of a full frame's pixels,
# with floor-saturating blobs, many discs and long scratches.
HEAVY_FRAME = DefectSpec(discs=9000, disc_radius=(1, 20), scratches=600,
                         scratch_length=(200, 4000), blobs=200)
# Fraction of a frame's pixels the NATIVE_FRAME defects touch (measured).
NATIVE_COVERAGE = 0.06
# Heavy damage at full size: about 5% of the pixels, most of it 200 blobs of
# radius U[20,60] whose IR keeps only 1-10% (scores saturate at the floor),
# plus long crossing scratches and some discs.
HEAVY_FULL = DefectSpec(discs=120, disc_radius=(1, 20), scratches=40,
                        scratch_length=(1000, 4000), blobs=200)


def scaled_spec(spec: DefectSpec, height: int, width: int) -> DefectSpec:
    """Scale defect counts by area relative to a full native frame."""

    area = height * width / float(FULL_FRAME[0] * FULL_FRAME[1])
    return DefectSpec(
        discs=max(1, int(round(spec.discs * area))),
        disc_radius=spec.disc_radius,
        scratches=max(1, int(round(spec.scratches * area))),
        scratch_length=spec.scratch_length,
        ir_factor=spec.ir_factor,
        rgb_factor=spec.rgb_factor,
        blobs=int(round(spec.blobs * area)),
        blob_radius=spec.blob_radius,
        blob_ir_factor=spec.blob_ir_factor,
    )


def _smooth_field(rng: np.random.Generator, height: int, width: int) -> np.ndarray:
    """Three 2-D sinusoids, evaluated as outer products (sin(a+b) expansion)."""

    field = np.zeros((height, width), np.float32)
    y = np.arange(height, dtype=np.float64) / height
    x = np.arange(width, dtype=np.float64) / width
    amplitudes = rng.dirichlet((2.0, 2.0, 2.0)) * 12000.0
    for amplitude in amplitudes:
        fy, fx = rng.uniform(0.5, 3.0, size=2) * rng.choice((-1.0, 1.0), size=2)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        a = 2.0 * np.pi * fy * y + phase
        b = 2.0 * np.pi * fx * x
        field += (amplitude * np.sin(a))[:, None].astype(np.float32) * np.cos(b)[None, :].astype(
            np.float32
        )
        field += (amplitude * np.cos(a))[:, None].astype(np.float32) * np.sin(b)[None, :].astype(
            np.float32
        )
    return field


def _disc_offsets(radius: float) -> tuple[np.ndarray, np.ndarray]:
    r = int(np.ceil(radius))
    dy, dx = np.mgrid[-r : r + 1, -r : r + 1]
    keep = dy * dy + dx * dx <= radius * radius + 1e-9
    return dy[keep], dx[keep]


def _apply(work: np.ndarray, ys: np.ndarray, xs: np.ndarray, ir: float, rgb: float) -> None:
    h, w = work.shape[:2]
    keep = (ys >= 0) & (ys < h) & (xs >= 0) & (xs < w)
    ys, xs = ys[keep], xs[keep]
    if ys.size == 0:
        return
    flat = np.unique(ys.astype(np.int64) * w + xs)
    ys, xs = flat // w, flat % w
    work[ys, xs, 3] *= np.float32(ir)
    work[ys, xs, :3] *= np.float32(rgb)


def _scratch_pixels(rng: np.random.Generator, height: int, width: int,
                    length: float) -> tuple[np.ndarray, np.ndarray]:
    vertices = int(rng.integers(2, 6))
    y0, x0 = rng.uniform(0, height), rng.uniform(0, width)
    heading = rng.uniform(0, 2 * np.pi)
    points = [(y0, x0)]
    step = length / (vertices - 1)
    for _ in range(vertices - 1):
        heading += rng.normal(0.0, 0.5)
        y0 += step * np.sin(heading)
        x0 += step * np.cos(heading)
        points.append((y0, x0))
    thickness = int(rng.integers(1, 4))
    if thickness == 1:
        oy, ox = np.zeros(1, np.int64), np.zeros(1, np.int64)
    else:
        oy, ox = _disc_offsets(thickness / 2.0)
    ys, xs = [], []
    for (ya, xa), (yb, xb) in zip(points[:-1], points[1:]):
        n = int(np.ceil(2 * np.hypot(yb - ya, xb - xa))) + 1
        t = np.linspace(0.0, 1.0, n)
        cy = np.rint(ya + (yb - ya) * t).astype(np.int64)
        cx = np.rint(xa + (xb - xa) * t).astype(np.int64)
        ys.append((cy[:, None] + oy[None, :]).ravel())
        xs.append((cx[:, None] + ox[None, :]).ravel())
    return np.concatenate(ys), np.concatenate(xs)


def make_frame(seed: int, height: int, width: int, spec: DefectSpec) -> np.ndarray:
    """One seeded HxWx4 uint16 RGBI main frame."""

    rng = np.random.default_rng(seed)
    work = np.empty((height, width, 4), np.float32)
    for c in range(3):
        work[:, :, c] = _smooth_field(rng, height, width)
        work[:, :, c] += np.float32(30000.0)
        work[:, :, c] += rng.normal(0.0, 600.0, size=(height, width)).astype(np.float32)
    work[:, :, 3] = np.float32(52000.0)
    work[:, :, 3] += rng.normal(0.0, 400.0, size=(height, width)).astype(np.float32)
    for _ in range(spec.discs):
        radius = rng.uniform(*spec.disc_radius)
        cy, cx = rng.uniform(0, height), rng.uniform(0, width)
        dy, dx = _disc_offsets(radius)
        _apply(work, int(cy) + dy, int(cx) + dx, rng.uniform(*spec.ir_factor),
               rng.uniform(*spec.rgb_factor))
    for _ in range(spec.scratches):
        ys, xs = _scratch_pixels(rng, height, width, rng.uniform(*spec.scratch_length))
        _apply(work, ys, xs, rng.uniform(*spec.ir_factor), rng.uniform(*spec.rgb_factor))
    for _ in range(spec.blobs):
        radius = rng.uniform(*spec.blob_radius)
        cy, cx = rng.uniform(0, height), rng.uniform(0, width)
        dy, dx = _disc_offsets(radius)
        _apply(work, int(cy) + dy, int(cx) + dx, rng.uniform(*spec.blob_ir_factor),
               rng.uniform(*spec.rgb_factor))
    np.clip(work, 0.0, 65535.0, out=work)
    return np.rint(work).astype(np.uint16)


def make_prepass(main: np.ndarray) -> np.ndarray:
    """Stride-14 decimation of the main frame (the 285 dpi prepass)."""

    return np.ascontiguousarray(main[::PREPASS_STRIDE, ::PREPASS_STRIDE])


def small_crop(seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """512x512 frame with 40 discs and 6 scratches."""

    main = make_frame(seed, 512, 512, SMALL_CROP)
    return main, make_prepass(main)


def native_frame(seed: int = 2, *, height: int = FULL_FRAME[0],
                 width: int = FULL_FRAME[1]) -> tuple[np.ndarray, np.ndarray]:
    """Full 4000 dpi frame (5782x3946 by default), ~0.5% defect coverage."""

    main = make_frame(seed, height, width, scaled_spec(NATIVE_FRAME, height, width))
    return main, make_prepass(main)


def heavy_frame(seed: int, *, height: int = FULL_FRAME[0],
                width: int = FULL_FRAME[1]) -> tuple[np.ndarray, np.ndarray]:
    """Heavy-damage frame (~5% coverage with floor-saturating blobs)."""

    main = make_frame(seed, height, width, scaled_spec(HEAVY_FRAME, height, width))
    return main, make_prepass(main)


def heavy_full_frame(index: int, base_seed: int = 200) -> tuple[np.ndarray, np.ndarray]:
    """Frame ``index`` of the heavy-damage batch: a full 5782x3946 frame at
    about 5% coverage (HEAVY_FULL), seed base+index."""

    main = make_frame(base_seed + index, FULL_FRAME[0], FULL_FRAME[1], HEAVY_FULL)
    return main, make_prepass(main)


def coverage_frame(seed: int, height: int, width: int, coverage: float) -> np.ndarray:
    """A frame from the native generator with its defect counts scaled to a
    target coverage, the fraction of pixels a defect touches: the serving
    workload draws each request's coverage from U[0.1%, 3%].  The native
    spec's counts touch about 6% of a frame (NATIVE_COVERAGE, measured on
    this generator), and coverage grows about linearly with the counts in
    this range."""

    base = scaled_spec(NATIVE_FRAME, height, width)
    factor = coverage / NATIVE_COVERAGE
    spec = DefectSpec(discs=max(1, int(round(base.discs * factor))),
                      disc_radius=base.disc_radius,
                      scratches=max(1, int(round(base.scratches * factor))),
                      scratch_length=base.scratch_length)
    return make_frame(seed, height, width, spec)


def crop_origins(height: int, width: int, size: int, count: int, base_seed: int = 1000):
    """Seeded crop origins: crop i uses default_rng(base_seed + i)."""

    origins = []
    for i in range(count):
        r = np.random.default_rng(base_seed + i)
        origins.append((int(r.integers(0, height - size + 1)), int(r.integers(0, width - size + 1))))
    return origins


# Batched workload: uneven sizes cycling through five shapes.
BATCH_SHAPES = ((5782, 3946), (3946, 5782), (2892, 1973), (1024, 768), (4000, 2700))


def batch_frame(index: int, base_seed: int = 100) -> tuple[np.ndarray, np.ndarray]:
    """Frame ``index`` of the batched workload (shape cycles, seed base+index)."""

    h, w = BATCH_SHAPES[index % len(BATCH_SHAPES)]
    main = make_frame(base_seed + index, h, w, scaled_spec(NATIVE_FRAME, h, w))
    return main, make_prepass(main)


def batch_frames(count: int = 16, base_seed: int = 100):
    """Frames of uneven sizes and orientations with per-frame seeds."""

    return [batch_frame(i, base_seed) for i in range(count)]
