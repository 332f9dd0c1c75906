"""At-floor routing census on the B200: the reference's routing contract.

Mirrors ``hybrid/src/fauxce_hybrid/routing.py`` (route_at_floor_mask,
:447-682; routing_json_document, :685-779; serialize_routing_json,
:782-793): the same policy object, reasons, dispositions, result tables,
errors and canonical JSON bytes.  Every per-pixel step runs in the library's
kernels (``fx_route.cu``): 8-connected labelling, chessboard distance,
per-label area / box / maximum, square dilation, the perimeter clear, the
oversized-region tiling, the overlap counts and the provisional/final pairs.
What stays on the host is per-component bookkeeping over K components
(reasons, routing decision, id ordering, the pair table) and the JSON.

There is no CPU fallback: without the library or a CUDA device the call
raises.
"""

from __future__ import annotations

import ctypes
import json
import math
import weakref
from dataclasses import dataclass
from enum import StrEnum
from fractions import Fraction

import numpy as np
import numpy.typing as npt

from . import _lib

BoolImage = npt.NDArray[np.bool_]
LabelImage = npt.NDArray[np.int32]

# Crop geometry of the inpainting call that consumes the final regions
# (routing.py:19-32): a final region whose bounding box, grown by the crop
# margin and clipped to the frame, covers more than MAX_INPAINT_CROP_PIXELS is
# split into MAX_SYNTHESIS_TILE_EDGE-sized grid tiles.
INPAINT_CROP_MARGIN = 128
MAX_INPAINT_CROP_PIXELS = 4_194_304
MAX_SYNTHESIS_TILE_EDGE = math.isqrt(MAX_INPAINT_CROP_PIXELS) - 2 * INPAINT_CROP_MARGIN

SCHEMA = "fauxce-hybrid-routing-v1"


class RoutedReason(StrEnum):
    """Threshold predicate(s) that route a region (routing.py:35-41)."""

    NOT_ROUTED = "not_routed"
    AREA = "area"
    CHESSBOARD_RADIUS = "chessboard_radius"
    AREA_AND_CHESSBOARD_RADIUS = "area+chessboard_radius"


class RegionDisposition(StrEnum):
    """How a provisional region relates to synthesis (routing.py:44-50)."""

    ROUTED = "routed"
    ABSORBED = "absorbed"
    PRISTINE = "pristine"
    PERIMETER_EXCLUDED = "perimeter_excluded"


class SynthesisBudgetExceeded(RuntimeError):
    """The routed mask exceeds its budget (routing.py:53-72)."""

    def __init__(self, *, synthesis_pixel_count: int, frame_pixel_count: int,
                 synthesis_fraction: float, maximum_fraction: float) -> None:
        self.synthesis_pixel_count = synthesis_pixel_count
        self.frame_pixel_count = frame_pixel_count
        self.synthesis_fraction = synthesis_fraction
        self.maximum_fraction = maximum_fraction
        super().__init__(
            "synthesis mask exceeds configured budget: "
            f"{synthesis_pixel_count}/{frame_pixel_count} pixels "
            f"({synthesis_fraction:.6%}) > {maximum_fraction:.6%}")


class NoHealthyContextError(RuntimeError):
    """The mask covers the whole frame (routing.py:75-85)."""

    def __init__(self, image_shape: tuple[int, int]) -> None:
        self.image_shape = image_shape
        self.finite_radius_sentinel = max(image_shape)
        super().__init__("at_floor_mask covers the entire frame; no healthy in-frame "
                         "context exists for bounded synthesis")


def _require_int(value: object, *, name: str, minimum: int) -> None:
    if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
        qualifier = "positive" if minimum == 1 else f">= {minimum}"
        raise ValueError(f"{name} must be a {qualifier} integer")


@dataclass(frozen=True)
class RoutingPolicy:
    """Thresholds and fail-closed budget (routing.py:94-117)."""

    min_area: int = 400
    min_radius: int = 5
    margin: int = 4
    max_synth_fraction: float = 0.02

    def __post_init__(self) -> None:
        _require_int(self.min_area, name="min_area", minimum=1)
        _require_int(self.min_radius, name="min_radius", minimum=1)
        _require_int(self.margin, name="margin", minimum=0)
        f = self.max_synth_fraction
        if (isinstance(f, bool) or not isinstance(f, (int, float))
                or not math.isfinite(float(f)) or not 0.0 <= float(f) <= 1.0):
            raise ValueError("max_synth_fraction must be finite and in [0, 1]")
        object.__setattr__(self, "max_synth_fraction", float(f))


@dataclass(frozen=True, order=True)
class BoundingBox:
    """Half-open ``[y0:y1, x0:x1]`` box (routing.py:119-140)."""

    y0: int
    x0: int
    y1: int
    x1: int

    def __post_init__(self) -> None:
        for name in ("y0", "x0", "y1", "x1"):
            _require_int(getattr(self, name), name=name, minimum=0)
        if self.y1 <= self.y0 or self.x1 <= self.x0:
            raise ValueError("bounding box must have positive half-open geometry")

    def as_list(self) -> list[int]:
        return [self.y0, self.x0, self.y1, self.x1]


@dataclass(frozen=True)
class ProvisionalRegion:
    """One 8-connected component of the at-floor mask (routing.py:143-158)."""

    id: int
    bbox: BoundingBox
    area: int
    max_chessboard_radius: int
    routed_reason: RoutedReason
    disposition: RegionDisposition
    final_component_ids: tuple[int, ...]
    absorbed_pixel_count: int

    @property
    def directly_routed(self) -> bool:
        return self.disposition is RegionDisposition.ROUTED


@dataclass(frozen=True)
class FinalSynthesisRegion:
    """One component of the dilated routed union (routing.py:161-170)."""

    id: int
    bbox: BoundingBox
    area: int
    direct_region_ids: tuple[int, ...]
    absorbed_region_ids: tuple[int, ...]
    non_floor_synth_pixel_count: int


def _check_plane(array: np.ndarray, *, name: str, dtype: np.dtype,
                 shape: tuple[int, int]) -> None:
    if array.dtype != dtype or array.shape != shape:
        raise ValueError(f"{name} must have dtype {dtype} and shape {shape}")
    if not array.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")
    if array.flags.writeable:
        raise ValueError(f"{name} must be read-only")


def _check_planes(result) -> None:
    _check_plane(result.provisional_labels, name="provisional_labels",
                 dtype=np.dtype(np.int32), shape=result.image_shape)
    _check_plane(result.synthesis_mask, name="synthesis_mask", dtype=np.dtype(np.bool_),
                 shape=result.image_shape)
    _check_plane(result.final_labels, name="final_labels", dtype=np.dtype(np.int32),
                 shape=result.image_shape)


@dataclass(frozen=True)
class RoutingResult:
    """Region tables and planes of one routing decision (routing.py:187-241)."""

    image_shape: tuple[int, int]
    policy: RoutingPolicy
    provisional_regions: tuple[ProvisionalRegion, ...]
    final_regions: tuple[FinalSynthesisRegion, ...]
    provisional_labels: LabelImage
    synthesis_mask: BoolImage
    final_labels: LabelImage
    at_floor_pixel_count: int
    directly_routed_pixel_count: int
    perimeter_excluded_region_count: int
    perimeter_excluded_pixel_count: int
    perimeter_suppressed_halo_pixel_count: int
    synthesis_pixel_count: int
    non_floor_synth_pixel_count: int
    synthesis_fraction: float
    within_synthesis_budget: bool

    def __post_init__(self) -> None:
        _check_planes(self)
        if not np.array_equal(self.final_labels > 0, self.synthesis_mask):
            raise ValueError("positive final labels must equal synthesis_mask")

    def require_safe_for_inpainting(self) -> None:
        """Raise before any model load when the budget is exceeded."""

        if not self.within_synthesis_budget:
            raise SynthesisBudgetExceeded(
                synthesis_pixel_count=self.synthesis_pixel_count,
                frame_pixel_count=self.image_shape[0] * self.image_shape[1],
                synthesis_fraction=self.synthesis_fraction,
                maximum_fraction=self.policy.max_synth_fraction)


def routed_reasons(areas: np.ndarray, radii: np.ndarray,
                   policy: RoutingPolicy) -> list[RoutedReason]:
    """Per-component reason from the two thresholds (routing.py:281-295)."""

    codes = (np.asarray(areas) >= policy.min_area).astype(np.int64) * 2 + (
        np.asarray(radii) >= policy.min_radius)
    return [_REASONS[c] for c in codes.tolist()]


def within_budget(synthesis_pixels: int, frame_pixels: int, maximum_fraction: float) -> bool:
    """Exact rational budget test on the fraction's decimal text
    (routing.py:315-322)."""

    limit = Fraction(str(maximum_fraction))
    return synthesis_pixels * limit.denominator <= frame_pixels * limit.numerator


def crop_pixels(boxes: np.ndarray, height: int, width: int) -> np.ndarray:
    """Pixels of each box grown by INPAINT_CROP_MARGIN and clipped to the
    frame (routing.py:343-348); boxes is K x 4 [y0, x0, y1, x1]."""

    b = boxes.astype(np.int64)
    y0 = np.maximum(0, b[:, 0] - INPAINT_CROP_MARGIN)
    x0 = np.maximum(0, b[:, 1] - INPAINT_CROP_MARGIN)
    y1 = np.minimum(height, b[:, 2] + INPAINT_CROP_MARGIN)
    x1 = np.minimum(width, b[:, 3] + INPAINT_CROP_MARGIN)
    return (y1 - y0) * (x1 - x0)


# ---------------------------------------------------------------------------
# Device side
# ---------------------------------------------------------------------------


class _Device:
    """Library calls on torch-owned device buffers, all on one stream."""

    def __init__(self) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("B200 routing requires a CUDA device; no CPU fallback exists")
        self.torch = torch
        self.lib = _lib.load()
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        self.err = torch.zeros(4, dtype=torch.int64, device=self.dev)  # err / flag / counter
        self.copy_stream = torch.cuda.Stream(device=self.dev)

    def download(self, t):
        """Start copying device tensor ``t`` (in its final state) into pinned
        host memory on the copy stream; the host tensor is valid after
        finish_downloads."""

        host = self.torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        ready = self.torch.cuda.Event()
        ready.record(self.torch.cuda.current_stream(self.dev))
        self.copy_stream.wait_event(ready)
        with self.torch.cuda.stream(self.copy_stream):
            host.copy_(t, non_blocking=True)
        return host

    def finish_downloads(self) -> None:
        self.copy_stream.synchronize()

    def empty(self, shape, dtype):
        return self.torch.empty(shape, dtype=dtype, device=self.dev)

    @staticmethod
    def p(t) -> ctypes.c_void_p | None:
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    def check(self, status: int, what: str) -> None:
        if status != 0:
            raise RuntimeError(f"{what} failed with library status {status}")

    def label8(self, mask_u8, h: int, w: int):
        t = self.torch
        labels = self.empty((h, w), t.int32)
        forest = self.empty((h, w), t.int32)
        scratch = self.empty(((h * w + 255) // 256 + 1,), t.int32)
        count = ctypes.c_int64()
        self.check(self.lib.fx_label8(self.p(mask_u8), h, w, self.p(labels), self.p(forest),
                                      self.p(scratch), self.p(self.err), ctypes.byref(count),
                                      self.stream), "fx_label8")
        return labels, int(count.value)

    def distance(self, mask_u8, h: int, w: int):
        t = self.torch
        dist = self.empty((h, w), t.int32)
        work = self.empty((h, w), t.int32)
        self.check(self.lib.fx_chessboard_distance(self.p(mask_u8), h, w, self.p(dist),
                                                   self.p(work), self.p(self.err), self.stream),
                   "fx_chessboard_distance")
        return dist

    def stats(self, labels, plane, h: int, w: int, k: int):
        """(areas int64[k], boxes int64[k, 4], maxima int64[k] or None) on the host."""

        t = self.torch
        if k == 0:
            return (np.zeros(0, np.int64), np.zeros((0, 4), np.int64),
                    None if plane is None else np.zeros(0, np.int64))
        area = self.empty((k,), t.int64)
        box = self.empty((k, 4), t.int32)
        vmax = self.empty((k,), t.int32) if plane is not None else None
        self.check(self.lib.fx_label_stats(self.p(labels), self.p(plane), h, w, k,
                                           self.p(area), self.p(box), self.p(vmax), self.stream),
                   "fx_label_stats")
        return (area.cpu().numpy().astype(np.int64), box.cpu().numpy().astype(np.int64),
                None if vmax is None else vmax.cpu().numpy().astype(np.int64))

    def map_labels(self, labels, table: np.ndarray, *, as_mask: bool):
        t = self.torch
        d_map = t.from_numpy(np.ascontiguousarray(table, dtype=np.int32)).to(self.dev)
        out = self.empty(tuple(labels.shape), t.uint8 if as_mask else t.int32)
        self.check(self.lib.fx_map_labels(
            self.p(labels), labels.numel(), self.p(d_map), len(table) - 1,
            None if as_mask else self.p(out), self.p(out) if as_mask else None, self.stream),
            "fx_map_labels")
        return out

    def dilate(self, mask_u8, h: int, w: int, radius: int):
        t = self.torch
        work = self.empty((h, w), t.uint8)
        out = self.empty((h, w), t.uint8)
        self.check(self.lib.fx_dilate_square(self.p(mask_u8), h, w, radius, self.p(work),
                                             self.p(out), self.stream), "fx_dilate_square")
        return out

    def clear_label(self, mask_u8, labels, label_id: int) -> int:
        cleared = ctypes.c_int64()
        self.check(self.lib.fx_clear_label(self.p(mask_u8), self.p(labels), labels.numel(),
                                           label_id, self.p(self.err), ctypes.byref(cleared),
                                           self.stream), "fx_clear_label")
        return int(cleared.value)

    def count_where(self, key, cond, k: int) -> np.ndarray:
        counts = self.empty((k + 1,), self.torch.int64)
        self.check(self.lib.fx_count_where(self.p(key), self.p(cond), key.numel(), k,
                                           self.p(counts), self.stream), "fx_count_where")
        return counts.cpu().numpy().astype(np.int64)

    def pairs(self, a, b, h: int, w: int) -> np.ndarray:
        """Distinct (a, b) label pairs, sorted by (a, b), as an M x 2 array."""

        capacity = 1 << 16
        for _ in range(2):
            buf = self.empty((capacity, 2), self.torch.int32)
            count = ctypes.c_int64()
            status = self.lib.fx_label_pairs(self.p(a), self.p(b), h, w, capacity, self.p(buf),
                                             self.p(self.err), ctypes.byref(count), self.stream)
            if status == 4 and count.value > capacity:  # FX_ERR_OUT_OF_MEMORY: grow once
                capacity = int(count.value)
                continue
            self.check(status, "fx_label_pairs")
            found = buf[: int(count.value)].cpu().numpy().astype(np.int64)
            return np.unique(found, axis=0) if found.size else found.reshape(0, 2)
        raise RuntimeError("fx_label_pairs: pair count changed between two identical passes")

    def tile_extract(self, labels, h, w, y0, x0, th, tw, label_id):
        tile = self.empty((th, tw), self.torch.uint8)
        self.check(self.lib.fx_tile_extract(self.p(labels), h, w, y0, x0, th, tw, label_id,
                                            self.p(tile), self.stream), "fx_tile_extract")
        return tile

    def tile_scatter(self, tile_labels, h, w, y0, x0, th, tw, base, plane) -> None:
        self.check(self.lib.fx_tile_scatter(self.p(tile_labels), h, w, y0, x0, th, tw, base,
                                            self.p(plane), self.stream), "fx_tile_scatter")


def validate_mask(at_floor_mask):
    """The mask as a bool numpy array or bool torch tensor with its shape,
    checked like routing.py:450-461 (TypeError for the dtype, ValueError for
    the shape)."""

    try:
        import torch
    except ImportError:  # pragma: no cover - torch is a dependency
        torch = None
    if torch is not None and isinstance(at_floor_mask, torch.Tensor):
        if at_floor_mask.dtype != torch.bool:
            raise TypeError("at_floor_mask must have dtype bool")
        shape = tuple(at_floor_mask.shape)
        mask = at_floor_mask
    else:
        mask = np.asarray(at_floor_mask)
        if mask.dtype != np.dtype(np.bool_):
            raise TypeError("at_floor_mask must have dtype bool")
        shape = mask.shape
    if len(shape) != 2:
        raise ValueError("at_floor_mask must have shape HxW")
    if shape[0] == 0 or shape[1] == 0:
        raise ValueError("at_floor_mask cannot have an empty dimension")
    if shape[0] * shape[1] >= 1 << 31:
        raise ValueError("at_floor_mask is limited to fewer than 2**31 pixels")
    return mask, int(shape[0]), int(shape[1])


def _device_mask(dev: _Device, mask):
    """A validated mask as a contiguous device uint8 plane."""

    t = dev.torch
    if isinstance(mask, t.Tensor):
        return mask.to(dev.dev).contiguous().view(t.uint8)
    return t.from_numpy(np.ascontiguousarray(mask).view(np.uint8)).to(dev.dev)


def _perimeter_component(dev: _Device, labels) -> int | None:
    """The component holding every frame-perimeter pixel (routing.py:298-312)."""

    t = dev.torch
    edges = t.cat([labels[0, :], labels[-1, :], labels[:, 0], labels[:, -1]]).cpu().numpy()
    candidate = int(edges[0])
    if candidate == 0 or not np.all(edges == candidate):
        return None
    return candidate


def _final_labels(dev: _Device, synthesis_u8, h: int, w: int):
    """Final labels and boxes in the reference's order (routing.py:325-444):
    8-connected components of the synthesis mask; a component whose crop is
    too large splits into grid tiles of MAX_SYNTHESIS_TILE_EDGE, relabelled
    inside each tile; fragments are numbered in discovery order and sorted by
    (y0, x0, y1, x1, fragment id)."""

    raw, count = dev.label8(synthesis_u8, h, w)
    if count == 0:
        return raw, np.zeros((0, 4), np.int64)
    _, raw_boxes, _ = dev.stats(raw, None, h, w, count)
    oversized = crop_pixels(raw_boxes, h, w) > MAX_INPAINT_CROP_PIXELS
    if not oversized.any():
        order = np.lexsort((np.arange(count), raw_boxes[:, 3], raw_boxes[:, 2],
                            raw_boxes[:, 1], raw_boxes[:, 0]))
        table = np.zeros(count + 1, np.int32)
        table[order + 1] = np.arange(1, count + 1, dtype=np.int32)
        return dev.map_labels(raw, table, as_mask=False), raw_boxes[order]

    # fragment ids in discovery order: whole components take one id, an
    # oversized component takes one per connected piece of each tile
    fragment_of_raw = np.zeros(count + 1, np.int32)
    boxes: list[np.ndarray] = []
    pending: list[tuple] = []  # (raw id, tile origin and size, first fragment id)
    nxt = 1
    for raw_id in range(1, count + 1):
        box = raw_boxes[raw_id - 1]
        if not oversized[raw_id - 1]:
            fragment_of_raw[raw_id] = nxt
            boxes.append(box)
            nxt += 1
            continue
        ry0, rx0, ry1, rx1 = (int(v) for v in box)
        for y0 in range(ry0, ry1, MAX_SYNTHESIS_TILE_EDGE):
            y1 = min(y0 + MAX_SYNTHESIS_TILE_EDGE, ry1)
            for x0 in range(rx0, rx1, MAX_SYNTHESIS_TILE_EDGE):
                x1 = min(x0 + MAX_SYNTHESIS_TILE_EDGE, rx1)
                tile = dev.tile_extract(raw, h, w, y0, x0, y1 - y0, x1 - x0, raw_id)
                tile_labels, tile_count = dev.label8(tile, y1 - y0, x1 - x0)
                if tile_count == 0:
                    continue
                _, tile_boxes, _ = dev.stats(tile_labels, None, y1 - y0, x1 - x0, tile_count)
                tile_boxes = tile_boxes + np.array([y0, x0, y0, x0], np.int64)
                boxes.extend(tile_boxes)
                pending.append((tile_labels, y0, x0, y1 - y0, x1 - x0, nxt - 1))
                nxt += tile_count
    fragments = dev.map_labels(raw, fragment_of_raw, as_mask=False)
    for tile_labels, y0, x0, th, tw, base in pending:
        dev.tile_scatter(tile_labels, h, w, y0, x0, th, tw, base, fragments)
    total = nxt - 1
    frag_boxes = np.asarray(boxes, np.int64).reshape(total, 4)
    order = np.lexsort((np.arange(total), frag_boxes[:, 3], frag_boxes[:, 2],
                        frag_boxes[:, 1], frag_boxes[:, 0]))
    table = np.zeros(total + 1, np.int32)
    table[order + 1] = np.arange(1, total + 1, dtype=np.int32)
    return dev.map_labels(fragments, table, as_mask=False), frag_boxes[order]


def _read_only(array: np.ndarray) -> np.ndarray:
    array = np.ascontiguousarray(array)
    array.setflags(write=False)
    return array


_REASONS = (RoutedReason.NOT_ROUTED, RoutedReason.CHESSBOARD_RADIUS, RoutedReason.AREA,
            RoutedReason.AREA_AND_CHESSBOARD_RADIUS)
_ROUTED, _ABSORBED, _PRISTINE, _EXCLUDED = 0, 1, 2, 3
_DISPOSITIONS = (RegionDisposition.ROUTED, RegionDisposition.ABSORBED,
                 RegionDisposition.PRISTINE, RegionDisposition.PERIMETER_EXCLUDED)
_new = object.__new__


def _box(y0: int, x0: int, y1: int, x1: int) -> BoundingBox:
    """A BoundingBox from device-measured extents (valid by construction)."""

    b = _new(BoundingBox)
    d = b.__dict__
    d["y0"], d["x0"], d["y1"], d["x1"] = y0, x0, y1, x1
    return b


def _grouped(keys: np.ndarray, values: np.ndarray, count: int):
    """values split by key 1..count (keys sorted ascending): the per-key
    tuples, and the count + 1 offsets of the key ranges."""

    offsets = np.searchsorted(keys, np.arange(1, count + 2)).astype(np.int64)
    bounds, vals = offsets.tolist(), values.tolist()
    return [tuple(vals[bounds[i]:bounds[i + 1]]) for i in range(count)], offsets


def route_at_floor_mask(at_floor_mask, policy: RoutingPolicy = RoutingPolicy()) -> RoutingResult:
    """Measure and route an at-floor mask (routing.py:447-682) on the GPU.

    ``at_floor_mask`` is an HxW bool array, or a bool torch tensor (a device
    tensor stays on the device).  Same errors as the reference: TypeError for
    a wrong policy or dtype, ValueError for a wrong shape,
    NoHealthyContextError for an all-true mask.
    """

    if not isinstance(policy, RoutingPolicy):
        raise TypeError("policy must be a RoutingPolicy")
    host_mask, height, width = validate_mask(at_floor_mask)
    n = height * width
    dev = _Device()
    mask = _device_mask(dev, host_mask)

    prov, k = dev.label8(mask, height, width)
    dist = dev.distance(mask, height, width)
    areas, boxes, radii = dev.stats(prov, dist, height, width, k)
    if int(areas.sum()) == n:
        raise NoHealthyContextError((height, width))
    prov_host = dev.download(prov)  # overlaps the rest of the census

    codes = (areas >= policy.min_area).astype(np.int64) * 2 + (radii >= policy.min_radius)
    perimeter_id = _perimeter_component(dev, prov)
    direct = codes != 0
    if perimeter_id is not None:
        direct[perimeter_id - 1] = False
    routed_table = np.zeros(k + 1, np.int32)
    routed_table[1:] = direct
    synthesis = dev.map_labels(prov, routed_table, as_mask=True)
    if policy.margin:
        synthesis = dev.dilate(synthesis, height, width, policy.margin)
    halo = 0
    if perimeter_id is not None:
        halo = dev.clear_label(synthesis, prov, perimeter_id)
    synthesis_host = dev.download(synthesis)

    final, final_boxes = _final_labels(dev, synthesis, height, width)
    final_host = dev.download(final)
    final_count = len(final_boxes)
    final_areas, check_boxes, _ = dev.stats(final, None, height, width, final_count)
    if not np.array_equal(check_boxes, final_boxes):
        raise RuntimeError("final label boxes disagree with their fragments")

    # overlap accounting (routing.py:528-556): per-region synthesised at-floor
    # pixels, per-final at-floor pixels, and the distinct (region, final) pairs
    overlap = dev.count_where(prov, final, k)
    final_floor = dev.count_where(final, prov, final_count)
    pairs = dev.pairs(prov, final, height, width)     # sorted by (region, final)
    pids, fids = pairs[:, 0], pairs[:, 1]
    if perimeter_id is not None and (np.any(pids == perimeter_id) or overlap[perimeter_id]):
        raise RuntimeError("perimeter-excluded region entered synthesis mask")
    synthesised = overlap[1:]
    disposition = np.where(direct, _ROUTED, np.where(synthesised > 0, _ABSORBED, _PRISTINE))
    if perimeter_id is not None:
        disposition[perimeter_id - 1] = _EXCLUDED
    final_ids, final_offsets = _grouped(pids, fids, k)
    if direct.any() and not np.all(np.isin(np.flatnonzero(direct) + 1, pids)):
        raise RuntimeError("directly routed region lost its final binding")
    by_final = np.lexsort((pids, fids))                # (final, region) order
    direct_pair = direct[pids[by_final] - 1]
    direct_vals, absorbed_vals = pids[by_final][direct_pair], pids[by_final][~direct_pair]
    direct_ids, direct_offsets = _grouped(fids[by_final][direct_pair], direct_vals, final_count)
    absorbed_ids, absorbed_offsets = _grouped(fids[by_final][~direct_pair], absorbed_vals,
                                              final_count)
    absorbed = np.where(disposition == _ABSORBED, synthesised, 0)

    regions = []
    box_rows, area_l, radius_l = boxes.tolist(), areas.tolist(), radii.tolist()
    code_l, disp_l, absorbed_l = codes.tolist(), disposition.tolist(), absorbed.tolist()
    for i in range(k):
        r = _new(ProvisionalRegion)
        r.__dict__.update(id=i + 1, bbox=_box(*box_rows[i]), area=area_l[i],
                          max_chessboard_radius=radius_l[i], routed_reason=_REASONS[code_l[i]],
                          disposition=_DISPOSITIONS[disp_l[i]], final_component_ids=final_ids[i],
                          absorbed_pixel_count=absorbed_l[i])
        regions.append(r)
    finals = []
    fbox_rows, farea_l = final_boxes.tolist(), final_areas.tolist()
    ffloor_l = final_floor.tolist()
    for f in range(final_count):
        r = _new(FinalSynthesisRegion)
        r.__dict__.update(id=f + 1, bbox=_box(*fbox_rows[f]), area=farea_l[f],
                          direct_region_ids=direct_ids[f], absorbed_region_ids=absorbed_ids[f],
                          non_floor_synth_pixel_count=farea_l[f] - ffloor_l[f + 1])
        finals.append(r)

    at_floor = int(areas.sum())
    directly_routed = int(areas[disposition == _ROUTED].sum())
    absorbed_total = int(absorbed.sum())
    synthesis_pixels = int(final_areas.sum())
    non_floor = synthesis_pixels - int(synthesised.sum())
    if synthesis_pixels != directly_routed + absorbed_total + non_floor:
        raise RuntimeError("synthesis pixel accounting is not conservative")

    dev.finish_downloads()
    fields = dict(
        image_shape=(height, width), policy=policy, provisional_regions=tuple(regions),
        final_regions=tuple(finals),
        provisional_labels=_read_only(prov_host.numpy()),
        synthesis_mask=_read_only(synthesis_host.numpy().view(np.bool_)),
        final_labels=_read_only(final_host.numpy()),
        at_floor_pixel_count=at_floor, directly_routed_pixel_count=directly_routed,
        perimeter_excluded_region_count=int(perimeter_id is not None),
        perimeter_excluded_pixel_count=(int(areas[perimeter_id - 1])
                                        if perimeter_id is not None else 0),
        perimeter_suppressed_halo_pixel_count=halo, synthesis_pixel_count=synthesis_pixels,
        non_floor_synth_pixel_count=non_floor, synthesis_fraction=synthesis_pixels / n,
        within_synthesis_budget=within_budget(synthesis_pixels, n, policy.max_synth_fraction))
    # The planes' dtype, shape, contiguity and read-only flags are checked as
    # in the constructor; the full-plane (final_labels > 0) == synthesis_mask
    # comparison is skipped because it holds by construction (the final
    # labels are the labelling of the synthesis mask), and the GPU tests
    # compare both planes with the oracle's.
    result = _new(RoutingResult)
    result.__dict__.update(fields)
    _check_planes(result)
    _attach_tables(result, _CensusTables(
        boxes=np.ascontiguousarray(boxes, np.int64), areas=areas.astype(np.int64),
        radii=radii.astype(np.int64), reasons=codes.astype(np.int32),
        dispositions=disposition.astype(np.int32), absorbed=absorbed.astype(np.int64),
        final_offsets=final_offsets, final_ids=np.ascontiguousarray(fids, np.int64),
        final_boxes=np.ascontiguousarray(final_boxes, np.int64),
        final_areas=final_areas.astype(np.int64), direct_offsets=direct_offsets,
        direct_ids=np.ascontiguousarray(direct_vals, np.int64), absorbed_offsets=absorbed_offsets,
        absorbed_ids=np.ascontiguousarray(absorbed_vals, np.int64),
        non_floor=(final_areas - final_floor[1:]).astype(np.int64)))
    return result


@dataclass(frozen=True)
class _CensusTables:
    """Flat region tables of a device-built result, for the native JSON writer."""

    boxes: np.ndarray
    areas: np.ndarray
    radii: np.ndarray
    reasons: np.ndarray
    dispositions: np.ndarray
    absorbed: np.ndarray
    final_offsets: np.ndarray
    final_ids: np.ndarray
    final_boxes: np.ndarray
    final_areas: np.ndarray
    direct_offsets: np.ndarray
    direct_ids: np.ndarray
    absorbed_offsets: np.ndarray
    absorbed_ids: np.ndarray
    non_floor: np.ndarray


# Tables of live device-built results, by id(result); an entry goes when its
# result is collected.  Results built any other way are serialized from
# their region objects.
_TABLES: dict[int, _CensusTables] = {}


def _attach_tables(result: RoutingResult, tables: _CensusTables) -> None:
    key = id(result)
    _TABLES[key] = tables
    weakref.finalize(result, _TABLES.pop, key, None)


def routing_json_document(result: RoutingResult) -> dict[str, object]:
    """The versioned routing census document (routing.py:685-779)."""

    if not isinstance(result, RoutingResult):
        raise TypeError("result must be a RoutingResult")
    doc = _document_head(result)
    doc["provisional_regions"] = [
        {
            "id": r.id,
            "bbox_yxyx_half_open": r.bbox.as_list(),
            "area": r.area,
            "max_chessboard_radius": r.max_chessboard_radius,
            "routed_reason": r.routed_reason.value,
            "disposition": r.disposition.value,
            "final_component_ids": list(r.final_component_ids),
            "absorbed_pixel_count": r.absorbed_pixel_count,
        }
        for r in result.provisional_regions
    ]
    doc["final_regions"] = [
        {
            "id": r.id,
            "bbox_yxyx_half_open": r.bbox.as_list(),
            "area": r.area,
            "direct_region_ids": list(r.direct_region_ids),
            "absorbed_region_ids": list(r.absorbed_region_ids),
            "non_floor_synthesis_pixels": r.non_floor_synth_pixel_count,
        }
        for r in result.final_regions
    ]
    return doc


def _document_head(result: RoutingResult) -> dict[str, object]:
    """Every key of the census document except the two region lists."""

    excluded = next((r for r in result.provisional_regions
                     if r.disposition is RegionDisposition.PERIMETER_EXCLUDED), None)
    height, width = result.image_shape
    perimeter_pixels = (width if height == 1 else height if width == 1
                        else 2 * (height + width) - 4)
    policy = result.policy
    return {
        "schema": SCHEMA,
        "image_shape": [height, width],
        "policy": {
            "connectivity": 8,
            "distance_metric": "chessboard",
            "distance_border_semantics": "unpadded_in_frame_background",
            "min_area": policy.min_area,
            "min_radius": policy.min_radius,
            "margin": policy.margin,
            "dilation": "single_square_chebyshev_footprint",
            "max_synth_fraction": policy.max_synth_fraction,
            "thresholds_provisional": True,
            "perimeter_rule": "exclude_component_covering_full_perimeter",
            "final_id_sort_key": ["y0", "x0", "y1", "x1", "raw_id"],
            "final_component_partition": {
                "algorithm": "bbox_grid_8_connected_fragments",
                "crop_margin": INPAINT_CROP_MARGIN,
                "max_crop_pixels": MAX_INPAINT_CROP_PIXELS,
                "max_core_tile_edge": MAX_SYNTHESIS_TILE_EDGE,
            },
        },
        "counts": {
            "frame_pixels": height * width,
            "at_floor_pixels": result.at_floor_pixel_count,
            "directly_routed_pixels": result.directly_routed_pixel_count,
            "perimeter_excluded_regions": result.perimeter_excluded_region_count,
            "perimeter_excluded_pixels": result.perimeter_excluded_pixel_count,
            "perimeter_suppressed_halo_pixels": result.perimeter_suppressed_halo_pixel_count,
            "provisional_regions": len(result.provisional_regions),
            "final_regions": len(result.final_regions),
            "synthesis_pixels": result.synthesis_pixel_count,
            "non_floor_synthesis_pixels": result.non_floor_synth_pixel_count,
        },
        "synthesis_fraction": result.synthesis_fraction,
        "within_synthesis_budget": result.within_synthesis_budget,
        "perimeter_excluded_region": None if excluded is None else {
            "id": excluded.id,
            "bbox_yxyx_half_open": excluded.bbox.as_list(),
            "area": excluded.area,
            "max_chessboard_radius": excluded.max_chessboard_radius,
            "routed_reason_by_thresholds": excluded.routed_reason.value,
            "perimeter_pixel_count": perimeter_pixels,
            "predicate": "contains_every_frame_perimeter_pixel",
            "content_interpretation": "unverified",
        },
    }


def _dumps(doc: dict) -> bytes:
    return json.dumps(doc, ensure_ascii=False, allow_nan=False, sort_keys=True,
                      separators=(",", ":")).encode("utf-8")


_PROVISIONAL_MARK, _FINAL_MARK = "@@provisional_regions@@", "@@final_regions@@"


def _native_lists(tables: _CensusTables) -> tuple[bytes, bytes]:
    """The two region lists written by the library from the flat tables."""

    lib = _lib.load()
    p = _lib.ptr
    k, f = len(tables.areas), len(tables.final_areas)
    cap = 256 + k * 330 + 21 * len(tables.final_ids)
    buf = np.empty(cap, np.uint8)
    n = lib.fx_census_provisional_json(
        k, p(tables.boxes), p(tables.areas), p(tables.radii), p(tables.reasons),
        p(tables.dispositions), p(tables.absorbed), p(tables.final_offsets), p(tables.final_ids),
        p(buf), cap)
    if n < 0:
        raise RuntimeError("fx_census_provisional_json failed")
    provisional = buf[:n].tobytes()
    cap = 256 + f * 250 + 21 * (len(tables.direct_ids) + len(tables.absorbed_ids))
    buf = np.empty(cap, np.uint8)
    n = lib.fx_census_final_json(
        f, p(tables.final_boxes), p(tables.final_areas), p(tables.direct_offsets),
        p(tables.direct_ids), p(tables.absorbed_offsets), p(tables.absorbed_ids),
        p(tables.non_floor), p(buf), cap)
    if n < 0:
        raise RuntimeError("fx_census_final_json failed")
    return provisional, buf[:n].tobytes()


def serialize_routing_json(result: RoutingResult) -> bytes:
    """Canonical UTF-8 JSON of the census (routing.py:782-793).

    For a result of route_at_floor_mask the two region lists are written by
    the library from the result's flat tables (same bytes, one pass); other
    results are serialized from their region objects."""

    if not isinstance(result, RoutingResult):
        raise TypeError("result must be a RoutingResult")
    tables = _TABLES.get(id(result))
    if tables is None:
        return _dumps(routing_json_document(result)) + b"\n"
    head = _document_head(result)
    head["provisional_regions"], head["final_regions"] = _PROVISIONAL_MARK, _FINAL_MARK
    provisional, final = _native_lists(tables)
    text = _dumps(head)
    text = text.replace(b'"' + _PROVISIONAL_MARK.encode() + b'"', provisional, 1)
    text = text.replace(b'"' + _FINAL_MARK.encode() + b'"', final, 1)
    return text + b"\n"


__all__ = [
    "BoundingBox", "FinalSynthesisRegion", "INPAINT_CROP_MARGIN", "MAX_INPAINT_CROP_PIXELS",
    "MAX_SYNTHESIS_TILE_EDGE", "NoHealthyContextError", "ProvisionalRegion",
    "RegionDisposition", "RoutedReason", "RoutingPolicy", "RoutingResult",
    "SynthesisBudgetExceeded", "route_at_floor_mask", "routing_json_document",
    "serialize_routing_json",
]
