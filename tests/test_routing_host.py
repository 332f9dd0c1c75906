"""At-floor routing census on the CPU: the oracle pinned to the reference,
and the host side of the device path (policy, validation, reasons, budget,
census document) checked without a GPU.

The golden file holds the reference's results on the masks of
golden/route_cases.py (golden/make_routing_golden.py).
"""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

import route_cases
from fauxice_b200 import routing
from oracle import routing_oracle as ro

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def route_golden():
    with open(os.path.join(HERE, "golden", "routing_golden.json")) as handle:
        return json.load(handle)["cases"]


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def _read_only(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    a.setflags(write=False)
    return a


def result_from_oracle(mask: np.ndarray, policy: routing.RoutingPolicy) -> routing.RoutingResult:
    """The oracle's census rebuilt as the product's result objects."""

    doc, prov, synth, final = ro.route(mask, **route_cases_policy(policy))
    c = doc["counts"]
    box = lambda b: routing.BoundingBox(*b)  # noqa: E731
    regions = tuple(
        routing.ProvisionalRegion(
            id=r["id"], bbox=box(r["bbox_yxyx_half_open"]), area=r["area"],
            max_chessboard_radius=r["max_chessboard_radius"],
            routed_reason=routing.RoutedReason(r["routed_reason"]),
            disposition=routing.RegionDisposition(r["disposition"]),
            final_component_ids=tuple(r["final_component_ids"]),
            absorbed_pixel_count=r["absorbed_pixel_count"])
        for r in doc["provisional_regions"])
    finals = tuple(
        routing.FinalSynthesisRegion(
            id=r["id"], bbox=box(r["bbox_yxyx_half_open"]), area=r["area"],
            direct_region_ids=tuple(r["direct_region_ids"]),
            absorbed_region_ids=tuple(r["absorbed_region_ids"]),
            non_floor_synth_pixel_count=r["non_floor_synthesis_pixels"])
        for r in doc["final_regions"])
    return routing.RoutingResult(
        image_shape=tuple(doc["image_shape"]), policy=policy, provisional_regions=regions,
        final_regions=finals, provisional_labels=_read_only(prov),
        synthesis_mask=_read_only(synth), final_labels=_read_only(final),
        at_floor_pixel_count=c["at_floor_pixels"],
        directly_routed_pixel_count=c["directly_routed_pixels"],
        perimeter_excluded_region_count=c["perimeter_excluded_regions"],
        perimeter_excluded_pixel_count=c["perimeter_excluded_pixels"],
        perimeter_suppressed_halo_pixel_count=c["perimeter_suppressed_halo_pixels"],
        synthesis_pixel_count=c["synthesis_pixels"],
        non_floor_synth_pixel_count=c["non_floor_synthesis_pixels"],
        synthesis_fraction=doc["synthesis_fraction"],
        within_synthesis_budget=doc["within_synthesis_budget"])


def route_cases_policy(policy: routing.RoutingPolicy) -> dict:
    return {"min_area": policy.min_area, "min_radius": policy.min_radius,
            "margin": policy.margin, "max_synth_fraction": policy.max_synth_fraction}


@pytest.mark.parametrize("name", list(route_cases.CASES))
def test_oracle_matches_reference(name, route_golden):
    expected = route_golden[name]
    mask = route_cases.mask(name)
    assert sha(mask.tobytes()) == expected["mask_sha256"]
    if "error" in expected:
        assert expected["error"] == "NoHealthyContextError"
        with pytest.raises(ro.NoHealthyContext):
            ro.route(mask, **route_cases.policy_kwargs(name))
        return
    doc, prov, synth, final = ro.route(mask, **route_cases.policy_kwargs(name))
    assert sha(ro.serialize(doc)) == expected["json_sha256"]
    assert sha(prov.tobytes()) == expected["provisional_labels_sha256"]
    assert sha(synth.tobytes()) == expected["synthesis_mask_sha256"]
    assert sha(final.tobytes()) == expected["final_labels_sha256"]
    if "json" in expected:
        assert ro.serialize(doc).decode("utf-8") == expected["json"]


@pytest.mark.parametrize("name", [n for n in route_cases.CASES
                                  if not route_cases.CASES[n].get("slow")])
def test_census_document_matches_reference_bytes(name, route_golden):
    """The product's result objects and JSON serializer reproduce the
    reference's canonical bytes (tables from the oracle, no GPU)."""

    expected = route_golden[name]
    if "error" in expected:
        pytest.skip("the reference raised for this mask")
    policy = routing.RoutingPolicy(**route_cases.policy_kwargs(name))
    result = result_from_oracle(route_cases.mask(name), policy)
    assert sha(routing.serialize_routing_json(result)) == expected["json_sha256"]


_REASON_CODE = {"not_routed": 0, "chessboard_radius": 1, "area": 2, "area+chessboard_radius": 3}
_DISPOSITION_CODE = {"routed": 0, "absorbed": 1, "pristine": 2, "perimeter_excluded": 3}


def _offsets(lists):
    offsets = np.zeros(len(lists) + 1, np.int64)
    offsets[1:] = np.cumsum([len(v) for v in lists])
    values = np.array([x for v in lists for x in v], dtype=np.int64)
    return offsets, values


def tables_from_oracle(doc: dict) -> "routing._CensusTables":
    prov, fin = doc["provisional_regions"], doc["final_regions"]
    i64 = lambda v: np.array(v, dtype=np.int64).reshape(-1)  # noqa: E731
    final_offsets, final_ids = _offsets([r["final_component_ids"] for r in prov])
    direct_offsets, direct_ids = _offsets([r["direct_region_ids"] for r in fin])
    absorbed_offsets, absorbed_ids = _offsets([r["absorbed_region_ids"] for r in fin])
    return routing._CensusTables(
        boxes=np.array([r["bbox_yxyx_half_open"] for r in prov], np.int64).reshape(-1, 4),
        areas=i64([r["area"] for r in prov]), radii=i64([r["max_chessboard_radius"] for r in prov]),
        reasons=np.array([_REASON_CODE[r["routed_reason"]] for r in prov], np.int32),
        dispositions=np.array([_DISPOSITION_CODE[r["disposition"]] for r in prov], np.int32),
        absorbed=i64([r["absorbed_pixel_count"] for r in prov]),
        final_offsets=final_offsets, final_ids=final_ids,
        final_boxes=np.array([r["bbox_yxyx_half_open"] for r in fin], np.int64).reshape(-1, 4),
        final_areas=i64([r["area"] for r in fin]), direct_offsets=direct_offsets,
        direct_ids=direct_ids, absorbed_offsets=absorbed_offsets, absorbed_ids=absorbed_ids,
        non_floor=i64([r["non_floor_synthesis_pixels"] for r in fin]))


@pytest.mark.parametrize("name", [n for n in route_cases.CASES
                                  if not route_cases.CASES[n].get("slow")])
def test_native_region_writer_matches_reference_bytes(name, route_golden):
    """The library's region-list writer, fed flat tables, gives the
    reference's canonical bytes (host code: no GPU needed)."""

    expected = route_golden[name]
    if "error" in expected:
        pytest.skip("the reference raised for this mask")
    policy = routing.RoutingPolicy(**route_cases.policy_kwargs(name))
    mask = route_cases.mask(name)
    result = result_from_oracle(mask, policy)
    doc, *_ = ro.route(mask, **route_cases.policy_kwargs(name))
    routing._attach_tables(result, tables_from_oracle(doc))
    assert id(result) in routing._TABLES
    assert sha(routing.serialize_routing_json(result)) == expected["json_sha256"]
    key = id(result)
    del result
    assert key not in routing._TABLES  # the side table follows the result's lifetime


def test_native_writer_rejects_short_buffers_and_bad_codes():
    from fauxice_b200 import _lib

    lib = _lib.load()
    z = np.zeros(4, np.int64)
    offsets = np.zeros(2, np.int64)
    codes = np.zeros(1, np.int32)
    buf = np.empty(8, np.uint8)
    p = _lib.ptr
    assert lib.fx_census_provisional_json(1, p(z), p(z), p(z), p(codes), p(codes), p(z),
                                          p(offsets), p(z), p(buf), 8) == -1
    bad = np.array([7], np.int32)
    big = np.empty(4096, np.uint8)
    assert lib.fx_census_provisional_json(1, p(z), p(z), p(z), p(bad), p(codes), p(z),
                                          p(offsets), p(z), p(big), 4096) == -1
    assert lib.fx_census_final_json(0, None, None, None, None, None, None, None, p(big),
                                    4096) == 2
    assert big[:2].tobytes() == b"[]"


def test_budget_is_an_exact_rational_test():
    assert routing.within_budget(2, 100, 0.02)
    assert not routing.within_budget(3, 100, 0.02)
    assert not routing.within_budget(1, 49, 0.02)      # 1/49 > 0.02
    assert routing.within_budget(0, 100, 0.0)
    assert not routing.within_budget(1, 100, 0.0)
    assert routing.within_budget(10, 100, 0.1)          # decimal text 0.1, not the binary float


def test_reasons_and_crop_geometry():
    reasons = routing.routed_reasons(np.array([400, 399, 10, 500]), np.array([1, 5, 4, 9]),
                                     routing.RoutingPolicy())
    assert [r.value for r in reasons] == ["area", "chessboard_radius", "not_routed",
                                          "area+chessboard_radius"]
    assert routing.MAX_SYNTHESIS_TILE_EDGE == 1792
    boxes = np.array([[0, 0, 10, 10], [200, 300, 2000, 2100]])
    assert routing.crop_pixels(boxes, 3000, 3000).tolist() == [138 * 138, 2056 * 2056]


@pytest.mark.parametrize("kwargs", [
    {"min_area": 0}, {"min_area": True}, {"min_area": 2.0}, {"min_radius": 0},
    {"margin": -1}, {"max_synth_fraction": float("nan")}, {"max_synth_fraction": 1.5},
    {"max_synth_fraction": -0.1}, {"max_synth_fraction": True}, {"max_synth_fraction": "0.1"},
])
def test_invalid_policy_is_rejected(kwargs):
    with pytest.raises(ValueError):
        routing.RoutingPolicy(**kwargs)


def test_policy_normalises_fraction_to_float():
    assert isinstance(routing.RoutingPolicy(max_synth_fraction=1).max_synth_fraction, float)


@pytest.mark.parametrize("mask, error", [
    (np.zeros((4, 4), dtype=np.uint8), TypeError),
    (np.zeros((4,), dtype=np.bool_), ValueError),
    (np.zeros((2, 3, 4), dtype=np.bool_), ValueError),
    (np.zeros((0, 5), dtype=np.bool_), ValueError),
    (np.zeros((5, 0), dtype=np.bool_), ValueError),
])
def test_invalid_mask_is_rejected_before_the_device(mask, error):
    with pytest.raises(error):
        routing.route_at_floor_mask(mask)


def test_non_policy_object_is_rejected():
    with pytest.raises(TypeError):
        routing.route_at_floor_mask(np.zeros((4, 4), dtype=np.bool_), policy={"margin": 1})


def test_result_planes_must_be_read_only_and_consistent():
    policy = routing.RoutingPolicy(min_area=1, margin=0)
    result = result_from_oracle(route_cases.points(6, 6, ((1, 1),)), policy)
    writable = np.array(result.final_labels)
    with pytest.raises(ValueError, match="read-only"):
        routing.RoutingResult(**{**result.__dict__, "final_labels": writable})
    bad = np.zeros((6, 6), dtype=np.int32)
    bad.setflags(write=False)
    with pytest.raises(ValueError, match="synthesis_mask"):
        routing.RoutingResult(**{**result.__dict__, "final_labels": bad})


def test_budget_guard_raises_with_counts():
    policy = routing.RoutingPolicy(min_area=1, min_radius=100, margin=0)
    result = result_from_oracle(route_cases.points(10, 10, ((1, 1), (8, 8), (5, 5))), policy)
    assert not result.within_synthesis_budget
    with pytest.raises(routing.SynthesisBudgetExceeded, match="3/100 pixels"):
        result.require_safe_for_inpainting()


def test_no_cpu_fallback_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises((RuntimeError, OSError)):
        routing.route_at_floor_mask(np.zeros((8, 8), dtype=np.bool_))


@pytest.mark.parametrize("seed", range(12))
def test_native_region_writer_matches_json_on_random_tables(seed):
    """Random tables (empty and long id lists, large values): the library's
    region lists equal json.dumps of the same region dicts, canonical form."""

    rng = np.random.default_rng(seed)
    k, f = int(rng.integers(0, 60)), int(rng.integers(0, 25))
    big = np.iinfo(np.int64).max // 4
    reasons = ["not_routed", "chessboard_radius", "area", "area+chessboard_radius"]
    dispositions = ["routed", "absorbed", "pristine", "perimeter_excluded"]
    rand_ids = lambda n: sorted(rng.choice(10**6, size=n, replace=False).tolist())  # noqa: E731
    prov = [{"id": i + 1, "bbox_yxyx_half_open": rng.integers(0, big, 4).tolist(),
             "area": int(rng.integers(0, big)), "max_chessboard_radius": int(rng.integers(0, 10**9)),
             "routed_reason": reasons[int(rng.integers(0, 4))],
             "disposition": dispositions[int(rng.integers(0, 4))],
             "final_component_ids": rand_ids(int(rng.integers(0, 6))),
             "absorbed_pixel_count": int(rng.integers(0, big))} for i in range(k)]
    fin = [{"id": i + 1, "bbox_yxyx_half_open": rng.integers(0, big, 4).tolist(),
            "area": int(rng.integers(0, big)), "direct_region_ids": rand_ids(int(rng.integers(0, 5))),
            "absorbed_region_ids": rand_ids(int(rng.integers(0, 40))),
            "non_floor_synthesis_pixels": int(rng.integers(0, big))} for i in range(f)]
    tables = tables_from_oracle({"provisional_regions": prov, "final_regions": fin})
    provisional, final = routing._native_lists(tables)
    dumps = lambda v: ro.serialize(v)[:-1]  # noqa: E731  (canonical, no trailing newline)
    assert provisional == dumps(prov)
    assert final == dumps(fin)
