"""CPU restatement of the at-floor routing census (numpy, pure-Python loops).

TEST INFRASTRUCTURE ONLY.  The tests use this module as the parity checker
of the device routing path; the B200 product never imports it.

It restates ``hybrid/src/fauxce_hybrid/routing.py`` of the reference without
scipy: the reference takes its per-pixel steps from scipy.ndimage (label with
a 3x3 structure, distance_transform_cdt with the chessboard metric, maximum,
find_objects, maximum_filter1d), whose published definitions are restated
here from first principles:

* 8-connected labelling: union-find over horizontal runs; ids 1..K in raster
  order of each component's first pixel (the order scipy.ndimage.label
  assigns).
* chessboard distance of a set pixel to the nearest unset in-frame pixel:
  the number of 3x3 erosions it survives, with pixels outside the frame
  counted as set (so they never act as background).
* square dilation: a 1-D window maximum along columns, then along rows,
  zero outside the frame.

It is pinned against tests/golden/routing_golden.json (outputs of the
reference run on the recipes of tests/golden/route_cases.py).
"""

from __future__ import annotations

import json
import math
from fractions import Fraction

import numpy as np

CROP_MARGIN = 128                      # routing.py:27
MAX_CROP_PIXELS = 4_194_304            # routing.py:28
MAX_TILE_EDGE = math.isqrt(MAX_CROP_PIXELS) - 2 * CROP_MARGIN  # routing.py:29-31


class NoHealthyContext(Exception):
    """routing.py:75-85: the mask is all true."""


def label8(mask: np.ndarray) -> tuple[np.ndarray, int]:
    """8-connected components (scipy.ndimage.label, 3x3 structure)."""

    h, w = mask.shape
    runs: list[tuple[int, int, int]] = []       # (row, start, stop)
    row_runs: list[list[int]] = []
    for y in range(h):
        row = mask[y].astype(np.int8)
        edges = np.flatnonzero(np.diff(np.concatenate(([0], row, [0]))))
        ids = []
        for s, e in zip(edges[0::2].tolist(), edges[1::2].tolist()):
            ids.append(len(runs))
            runs.append((y, s, e))
        row_runs.append(ids)
    parent = list(range(len(runs)))

    def find(a: int) -> int:
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for y in range(1, h):
        above = row_runs[y - 1]
        j = 0
        for r in row_runs[y]:
            _, s, e = runs[r]
            # runs above that touch [s - 1, e] (diagonal contact included)
            while j < len(above) and runs[above[j]][2] < s:
                j += 1
            k = j
            while k < len(above) and runs[above[k]][1] <= e:
                a, b = find(r), find(above[k])
                if a != b:
                    parent[max(a, b)] = min(a, b)
                k += 1
    labels = np.zeros((h, w), dtype=np.int32)
    ids: dict[int, int] = {}
    for r, (y, s, e) in enumerate(runs):   # runs are in raster order
        root = find(r)
        if root not in ids:
            ids[root] = len(ids) + 1
        labels[y, s:e] = ids[root]
    return labels, len(ids)


def _erode_square(m: np.ndarray) -> np.ndarray:
    """3x3 erosion with out-of-frame pixels counted as set."""

    v = m.copy()
    v[1:] &= m[:-1]
    v[:-1] &= m[1:]
    out = v.copy()
    out[:, 1:] &= v[:, :-1]
    out[:, :-1] &= v[:, 1:]
    return out


def chessboard_distance(mask: np.ndarray) -> np.ndarray:
    """distance_transform_cdt(mask, metric="chessboard") on a mask with at
    least one unset pixel."""

    dist = np.zeros(mask.shape, dtype=np.int64)
    level = mask.copy()
    while level.any():
        dist += level
        level = _erode_square(level)
    return dist


def _window_max(m: np.ndarray, r: int, axis: int) -> np.ndarray:
    out = m.copy()
    n = m.shape[axis]
    for d in range(1, min(r, n - 1) + 1):
        if axis == 0:
            out[d:] |= m[:-d]
            out[:-d] |= m[d:]
        else:
            out[:, d:] |= m[:, :-d]
            out[:, :-d] |= m[:, d:]
    return out


def dilate_square(mask: np.ndarray, radius: int) -> np.ndarray:
    """Separable square dilation clipped to the frame (routing.py:304-336)."""

    return _window_max(_window_max(mask, radius, 0), radius, 1)


def _boxes(labels: np.ndarray, k: int) -> np.ndarray:
    boxes = np.zeros((k, 4), dtype=np.int64)
    if k == 0:
        return boxes
    ys, xs = np.nonzero(labels)
    ls = labels[ys, xs] - 1
    boxes[:, 0] = labels.shape[0]
    boxes[:, 1] = labels.shape[1]
    np.minimum.at(boxes[:, 0], ls, ys)
    np.minimum.at(boxes[:, 1], ls, xs)
    np.maximum.at(boxes[:, 2], ls, ys + 1)
    np.maximum.at(boxes[:, 3], ls, xs + 1)
    return boxes


def _reason(area: int, radius: int, min_area: int, min_radius: int) -> str:
    """routing.py:281-295."""

    a, r = area >= min_area, radius >= min_radius
    return ("area+chessboard_radius" if a and r else "area" if a
            else "chessboard_radius" if r else "not_routed")


def _final_labels(synth: np.ndarray) -> tuple[np.ndarray, list[list[int]]]:
    """routing.py:325-444: components, oversized ones tiled, sorted ids."""

    h, w = synth.shape
    raw, count = label8(synth)
    raw_boxes = _boxes(raw, count)
    boxes: list[list[int]] = []
    whole = np.zeros(count + 1, dtype=np.int32)   # fragment id of each untiled component
    tiled: list[tuple] = []
    for raw_id in range(1, count + 1):
        y0, x0, y1, x1 = raw_boxes[raw_id - 1].tolist()
        crop = ((min(h, y1 + CROP_MARGIN) - max(0, y0 - CROP_MARGIN))
                * (min(w, x1 + CROP_MARGIN) - max(0, x0 - CROP_MARGIN)))
        if crop <= MAX_CROP_PIXELS:
            whole[raw_id] = len(boxes) + 1
            boxes.append([y0, x0, y1, x1])
            continue
        for ty in range(y0, y1, MAX_TILE_EDGE):
            for tx in range(x0, x1, MAX_TILE_EDGE):
                ey, ex = min(ty + MAX_TILE_EDGE, y1), min(tx + MAX_TILE_EDGE, x1)
                tile, tcount = label8(raw[ty:ey, tx:ex] == raw_id)
                tiled.append((ty, ey, tx, ex, tile, len(boxes)))
                for by0, bx0, by1, bx1 in _boxes(tile, tcount).tolist():
                    boxes.append([ty + by0, tx + bx0, ty + by1, tx + bx1])
    fragments = whole[raw]
    for ty, ey, tx, ex, tile, base in tiled:
        view = fragments[ty:ey, tx:ex]
        view[tile > 0] = base + tile[tile > 0]
    order = sorted(range(len(boxes)), key=lambda i: (*boxes[i], i + 1))
    table = np.zeros(len(boxes) + 1, dtype=np.int32)
    for new, old in enumerate(order, start=1):
        table[old + 1] = new
    return table[fragments], [boxes[i] for i in order]


def route(mask: np.ndarray, *, min_area: int = 400, min_radius: int = 5, margin: int = 4,
          max_synth_fraction: float = 0.02):
    """(census document, provisional labels, synthesis mask, final labels)
    for one at-floor mask (routing.py:447-682 and :685-779)."""

    mask = np.ascontiguousarray(mask, dtype=np.bool_)
    h, w = mask.shape
    if mask.all():
        raise NoHealthyContext((h, w))
    prov, k = label8(mask)
    areas = np.bincount(prov.ravel(), minlength=k + 1)[1:].astype(np.int64)
    radii = np.zeros(k, dtype=np.int64)
    if k:
        dist = chessboard_distance(mask)
        np.maximum.at(radii, prov[mask] - 1, dist[mask])
    boxes = _boxes(prov, k)
    reasons = [_reason(int(a), int(r), min_area, min_radius) for a, r in zip(areas, radii)]
    c = int(prov[0, 0])
    edge = np.concatenate([prov[0, :], prov[-1, :], prov[:, 0], prov[:, -1]])
    perimeter = c if c and bool(np.all(edge == c)) else None
    direct = [reasons[i] != "not_routed" and i + 1 != perimeter for i in range(k)]

    routed = np.zeros(k + 1, dtype=np.bool_)
    routed[1:] = direct
    synth = routed[prov]
    if margin:
        synth = dilate_square(synth, margin)
    halo = 0
    if perimeter is not None:
        on_perimeter = prov == perimeter
        halo = int(np.count_nonzero(synth & on_perimeter))
        synth[on_perimeter] = False

    final, final_boxes = _final_labels(synth)
    nf = len(final_boxes)
    both = (final > 0) & (prov > 0)
    overlap = np.bincount(prov[both], minlength=k + 1)
    final_floor = np.bincount(final[both], minlength=nf + 1)
    final_area = np.bincount(final.ravel(), minlength=nf + 1)
    pairs = sorted(set(zip(prov[both].tolist(), final[both].tolist())))
    final_ids: list[list[int]] = [[] for _ in range(k)]
    direct_ids: list[list[int]] = [[] for _ in range(nf)]
    absorbed_ids: list[list[int]] = [[] for _ in range(nf)]
    for p, f in pairs:
        final_ids[p - 1].append(f)
        (direct_ids if direct[p - 1] else absorbed_ids)[f - 1].append(p)

    regions = []
    for i in range(1, k + 1):
        s = int(overlap[i])
        if i == perimeter:
            disp, absorbed = "perimeter_excluded", 0
        elif direct[i - 1]:
            disp, absorbed = "routed", 0
        elif s:
            disp, absorbed = "absorbed", s
        else:
            disp, absorbed = "pristine", 0
        regions.append({
            "id": i, "bbox_yxyx_half_open": boxes[i - 1].tolist(), "area": int(areas[i - 1]),
            "max_chessboard_radius": int(radii[i - 1]), "routed_reason": reasons[i - 1],
            "disposition": disp, "final_component_ids": final_ids[i - 1],
            "absorbed_pixel_count": absorbed})
    finals = [{
        "id": f, "bbox_yxyx_half_open": final_boxes[f - 1], "area": int(final_area[f]),
        "direct_region_ids": direct_ids[f - 1], "absorbed_region_ids": absorbed_ids[f - 1],
        "non_floor_synthesis_pixels": int(final_area[f] - final_floor[f])}
        for f in range(1, nf + 1)]

    n = h * w
    synth_pixels = int(np.count_nonzero(synth))
    limit = Fraction(str(float(max_synth_fraction)))
    excluded = None
    if perimeter is not None:
        r = regions[perimeter - 1]
        excluded = {
            "id": perimeter, "bbox_yxyx_half_open": r["bbox_yxyx_half_open"], "area": r["area"],
            "max_chessboard_radius": r["max_chessboard_radius"],
            "routed_reason_by_thresholds": r["routed_reason"],
            "perimeter_pixel_count": w if h == 1 else h if w == 1 else 2 * (h + w) - 4,
            "predicate": "contains_every_frame_perimeter_pixel",
            "content_interpretation": "unverified"}
    doc = {
        "schema": "fauxce-hybrid-routing-v1",
        "image_shape": [h, w],
        "policy": {
            "connectivity": 8, "distance_metric": "chessboard",
            "distance_border_semantics": "unpadded_in_frame_background",
            "min_area": min_area, "min_radius": min_radius, "margin": margin,
            "dilation": "single_square_chebyshev_footprint",
            "max_synth_fraction": float(max_synth_fraction), "thresholds_provisional": True,
            "perimeter_rule": "exclude_component_covering_full_perimeter",
            "final_id_sort_key": ["y0", "x0", "y1", "x1", "raw_id"],
            "final_component_partition": {
                "algorithm": "bbox_grid_8_connected_fragments", "crop_margin": CROP_MARGIN,
                "max_crop_pixels": MAX_CROP_PIXELS, "max_core_tile_edge": MAX_TILE_EDGE}},
        "counts": {
            "frame_pixels": n, "at_floor_pixels": int(areas.sum()),
            "directly_routed_pixels": sum(r["area"] for r in regions
                                          if r["disposition"] == "routed"),
            "perimeter_excluded_regions": int(perimeter is not None),
            "perimeter_excluded_pixels": int(areas[perimeter - 1]) if perimeter else 0,
            "perimeter_suppressed_halo_pixels": halo,
            "provisional_regions": k, "final_regions": nf,
            "synthesis_pixels": synth_pixels,
            "non_floor_synthesis_pixels": int(np.count_nonzero(synth & ~mask))},
        "synthesis_fraction": synth_pixels / n,
        "within_synthesis_budget": synth_pixels * limit.denominator <= n * limit.numerator,
        "perimeter_excluded_region": excluded,
        "provisional_regions": regions,
        "final_regions": finals,
    }
    return doc, prov, synth, final


def serialize(doc: dict) -> bytes:
    """Canonical bytes of a census document (routing.py:782-793)."""

    return json.dumps(doc, ensure_ascii=False, allow_nan=False, sort_keys=True,
                      separators=(",", ":")).encode("utf-8") + b"\n"
