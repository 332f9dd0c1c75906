"""Seeded at-floor masks for the routing census parity cases.

The routing step (hybrid routing.py:447-682) takes one HxW bool mask and a
policy.  These recipes build masks that reach every branch of it: routed by
area, by radius or both; unrouted regions absorbed by a neighbour's dilation
or left pristine; the full-perimeter exclusion with its suppressed halo;
regions touching the frame edge (in-frame distance semantics); single-row
and single-column frames; margin 0; an exceeded budget; final components
with nested boxes; an empty mask; an all-true mask; and one sparse component
whose crop is too large, so the final labels split into grid tiles.

``make_routing_golden.py`` runs the reference on these masks and records
the results in ``routing_golden.json``; the tests rebuild the masks here.
"""

from __future__ import annotations

import numpy as np


def _blobs(rng: np.random.Generator, h: int, w: int, count: int, rmax: int) -> np.ndarray:
    """Discs and squares of random size and place, plus sparse speckle."""

    mask = rng.random((h, w)) < 0.01
    for _ in range(count):
        cy, cx = int(rng.integers(0, h)), int(rng.integers(0, w))
        r = int(rng.integers(1, rmax + 1))
        y0, y1, x0, x1 = max(0, cy - r), min(h, cy + r + 1), max(0, cx - r), min(w, cx + r + 1)
        if rng.random() < 0.5:
            yy, xx = np.mgrid[y0:y1, x0:x1]
            mask[y0:y1, x0:x1] |= (yy - cy) ** 2 + (xx - cx) ** 2 <= r * r
        else:
            mask[y0:y1, x0:x1] = True
    return mask


def dust(seed: int, h: int, w: int, count: int = 24, rmax: int = 14) -> np.ndarray:
    return _blobs(np.random.default_rng(seed), h, w, count, rmax)


def perimeter_ring(seed: int, h: int, w: int, thickness: int = 3) -> np.ndarray:
    """A border covering the whole frame perimeter plus interior dust; some
    dust touches the border (joins the perimeter component) and some lies
    within the dilation margin of it (suppressed halo)."""

    mask = dust(seed, h, w, count=14, rmax=9)
    mask[:thickness, :] = True
    mask[-thickness:, :] = True
    mask[:, :thickness] = True
    mask[:, -thickness:] = True
    # a routed square 2 pixels inside the border: its dilation reaches the ring
    mask[thickness + 2:thickness + 24, thickness + 2:thickness + 24] = True
    mask[thickness + 1, :] = False
    mask[:, thickness + 1] = False
    return mask


def broken_ring(seed: int, h: int, w: int) -> np.ndarray:
    """A border with one gap: no component covers the full perimeter."""

    mask = perimeter_ring(seed, h, w)
    mask[h // 2, 0] = False
    return mask


def absorbed(h: int = 60, w: int = 70) -> np.ndarray:
    """One routed square with small unrouted specks around it: specks within
    the margin are absorbed, the far ones stay pristine."""

    mask = np.zeros((h, w), dtype=np.bool_)
    mask[20:42, 20:42] = True
    for y, x in ((17, 30), (44, 25), (30, 45), (10, 10), (55, 60), (18, 18), (50, 50)):
        mask[y, x] = True
    mask[44, 26] = True
    return mask


def edge_blobs(h: int = 40, w: int = 50) -> np.ndarray:
    """Regions cut by the frame edge: distances count in-frame background only."""

    mask = np.zeros((h, w), dtype=np.bool_)
    mask[0:12, 10:22] = True       # touches the top edge
    mask[20:31, 0:11] = True       # touches the left edge
    mask[h - 9:h, w - 14:w] = True  # bottom-right corner
    return mask


def nested(h: int = 30, w: int = 30) -> np.ndarray:
    """A plus shape inside an open square frame (margin 0 keeps them apart):
    nested boxes order by their top-left corner."""

    mask = np.zeros((h, w), dtype=np.bool_)
    mask[4, 4:26] = True
    mask[4:26, 4] = True
    mask[25, 4:26] = True
    mask[4:23, 25] = True
    mask[15, 6:24] = True
    mask[6:24, 15] = True
    return mask


def comb(h: int = 2200, w: int = 2300) -> np.ndarray:
    """One sparse connected comb whose crop exceeds the inpainting limit:
    the final labels split into grid tiles, and teeth cut by a tile edge
    become separate fragments."""

    mask = np.zeros((h, w), dtype=np.bool_)
    mask[100:103, 100:w - 100] = True
    for x in range(100, w - 100, 211):
        mask[100:h - 60, x:x + 3] = True
    mask[h - 300:h - 297, 100:900] = True
    rng = np.random.default_rng(8)
    ys, xs = rng.integers(0, h, 400), rng.integers(0, w, 400)
    mask[ys, xs] = True
    return mask


def near_all_true(h: int = 11, w: int = 13) -> np.ndarray:
    """Everything at the floor except one interior pixel: one region, which
    covers the perimeter and is excluded."""

    mask = np.ones((h, w), dtype=np.bool_)
    mask[4, 9] = False
    return mask


def points(h: int, w: int, coords) -> np.ndarray:
    mask = np.zeros((h, w), dtype=np.bool_)
    for y, x in coords:
        mask[y, x] = True
    return mask


def diagonal(h: int = 40, w: int = 40) -> np.ndarray:
    """Diagonal strokes (8-connected only) and a checkerboard patch: one
    component each, with radius 1 whatever their box."""

    mask = np.zeros((h, w), dtype=np.bool_)
    idx = np.arange(30)
    mask[idx + 2, idx + 5] = True
    mask[idx[:20] + 5, 30 - idx[:20]] = True
    yy, xx = np.mgrid[:10, :10]
    mask[28:38, 2:12] |= (yy + xx) % 2 == 0
    return mask


def dense_rect(h: int = 2100, w: int = 2150) -> np.ndarray:
    """One dense rectangle whose crop exceeds the limit: four grid tiles."""

    mask = np.zeros((h, w), dtype=np.bool_)
    mask[90:2010, 80:2070] = True
    return mask


_EXACT = ((1, 2), (6, 11), (8, 3))

CASES: dict[str, dict] = {
    "dust_96x128": {"mask": lambda: dust(1, 96, 128)},
    "dust_small_policy_97x61": {"mask": lambda: dust(2, 97, 61, count=12, rmax=6),
                                "policy": {"min_area": 30, "min_radius": 3, "margin": 2}},
    "dust_margin0_64x64": {"mask": lambda: dust(3, 64, 64), "policy": {"margin": 0}},
    "dust_large_margin_50x90": {"mask": lambda: dust(4, 50, 90, count=8, rmax=10),
                                "policy": {"margin": 200, "max_synth_fraction": 1.0}},
    "perimeter_ring_80x100": {"mask": lambda: perimeter_ring(5, 80, 100)},
    "broken_ring_80x100": {"mask": lambda: broken_ring(5, 80, 100)},
    "absorbed_60x70": {"mask": absorbed},
    "edge_blobs_40x50": {"mask": edge_blobs, "policy": {"min_area": 10000, "min_radius": 6}},
    "nested_margin0_30x30": {"mask": nested, "policy": {"margin": 0, "min_area": 5}},
    "budget_exceeded_64x64": {"mask": lambda: dust(6, 64, 64, count=30, rmax=12),
                              "policy": {"max_synth_fraction": 0.01}},
    "budget_fraction_text_64x64": {"mask": lambda: dust(7, 64, 64, count=6, rmax=8),
                                   "policy": {"max_synth_fraction": 0.1}},
    "row_1x200": {"mask": lambda: np.random.default_rng(9).random((1, 200)) < 0.4,
                  "policy": {"min_area": 3, "min_radius": 1}},
    "column_150x1": {"mask": lambda: np.random.default_rng(10).random((150, 1)) < 0.5,
                     "policy": {"min_area": 4}},
    "empty_16x16": {"mask": lambda: np.zeros((16, 16), dtype=np.bool_)},
    "single_pixel_1x1_false": {"mask": lambda: np.zeros((1, 1), dtype=np.bool_)},
    "all_true_8x8": {"mask": lambda: np.ones((8, 8), dtype=np.bool_)},
    "dense_noise_300x400": {"mask": lambda: np.random.default_rng(11).random((300, 400)) < 0.45,
                            "policy": {"min_area": 50}},
    "dust_600x800": {"mask": lambda: dust(12, 600, 800, count=160, rmax=20)},
    "near_all_true_11x13": {"mask": near_all_true},
    "diagonal_40x40": {"mask": diagonal, "policy": {"min_area": 25, "min_radius": 2}},
    "budget_exact_10x15": {"mask": lambda: points(10, 15, _EXACT),
                           "policy": {"min_area": 1, "min_radius": 100, "margin": 0}},
    "budget_over_10x15": {"mask": lambda: points(10, 15, _EXACT + ((5, 7),)),
                          "policy": {"min_area": 1, "min_radius": 100, "margin": 0}},
    "budget_rational_7x7": {"mask": lambda: points(7, 7, ((2, 4),)),
                            "policy": {"min_area": 1, "min_radius": 100, "margin": 0}},
    "budget_zero_empty_12x12": {"mask": lambda: np.zeros((12, 12), dtype=np.bool_),
                                "policy": {"max_synth_fraction": 0.0}},
    "comb_tiled_2200x2300": {"mask": comb, "slow": True},
    "dense_rect_tiled_2100x2150": {"mask": dense_rect, "slow": True,
                                   "policy": {"min_area": 1, "min_radius": 100, "margin": 0,
                                              "max_synth_fraction": 1.0}},
}


def policy_kwargs(name: str) -> dict:
    return dict(CASES[name].get("policy", {}))


def mask(name: str) -> np.ndarray:
    return np.ascontiguousarray(CASES[name]["mask"](), dtype=np.bool_)
