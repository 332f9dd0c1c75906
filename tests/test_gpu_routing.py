"""At-floor routing census on the B200: bit-identical to the reference.

Every golden mask goes through route_at_floor_mask on the device and must
give the reference's census bytes and planes; seeded random masks (ragged
sizes, single rows and columns, perimeter rings, full-frame size) must match
the oracle; each device primitive is checked against its oracle restatement.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import route_cases
from fauxice_b200 import _lib, routing
from oracle import routing_oracle as ro

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


@pytest.fixture(scope="module")
def route_golden():
    with open(os.path.join(HERE, "golden", "routing_golden.json")) as handle:
        return json.load(handle)["cases"]


@pytest.mark.parametrize("name", list(route_cases.CASES))
def test_device_census_matches_reference(name, route_golden):
    expected = route_golden[name]
    mask = route_cases.mask(name)
    policy = routing.RoutingPolicy(**route_cases.policy_kwargs(name))
    if "error" in expected:
        with pytest.raises(routing.NoHealthyContextError) as raised:
            routing.route_at_floor_mask(mask, policy)
        assert raised.value.image_shape == mask.shape
        assert raised.value.finite_radius_sentinel == max(mask.shape)
        return
    result = routing.route_at_floor_mask(mask, policy)
    payload = routing.serialize_routing_json(result)
    if "json" in expected and sha(payload) != expected["json_sha256"]:
        assert payload.decode("utf-8") == expected["json"]
    assert sha(payload) == expected["json_sha256"]
    assert sha(result.provisional_labels.tobytes()) == expected["provisional_labels_sha256"]
    assert sha(result.synthesis_mask.tobytes()) == expected["synthesis_mask_sha256"]
    assert sha(result.final_labels.tobytes()) == expected["final_labels_sha256"]
    for plane in (result.provisional_labels, result.synthesis_mask, result.final_labels):
        assert not plane.flags.writeable


def test_device_tensor_input_matches_host_input():
    import torch

    mask = route_cases.mask("perimeter_ring_80x100")
    host = routing.serialize_routing_json(routing.route_at_floor_mask(mask))
    device = routing.serialize_routing_json(
        routing.route_at_floor_mask(torch.from_numpy(mask).to("cuda")))
    assert host == device


def _random_mask(seed: int) -> tuple[np.ndarray, dict]:
    rng = np.random.default_rng(seed)
    kind = seed % 5
    if kind == 0:
        h, w = int(rng.integers(1, 4)), int(rng.integers(1, 700))
        m = rng.random((h, w)) < rng.uniform(0.1, 0.8)
    elif kind == 1:
        h, w = int(rng.integers(1, 700)), int(rng.integers(1, 4))
        m = rng.random((h, w)) < rng.uniform(0.1, 0.8)
    elif kind == 2:
        h, w = int(rng.integers(33, 400)), int(rng.integers(33, 400))
        m = route_cases.perimeter_ring(seed, h, w, thickness=int(rng.integers(1, 5)))
    elif kind == 3:
        h, w = int(rng.integers(40, 700)), int(rng.integers(40, 700))
        m = route_cases.dust(seed, h, w, count=int(rng.integers(1, 80)), rmax=20)
    else:
        h, w = int(rng.integers(20, 500)), int(rng.integers(20, 500))
        m = rng.random((h, w)) < rng.uniform(0.2, 0.6)
    policy = {"min_area": int(rng.integers(1, 500)), "min_radius": int(rng.integers(1, 8)),
              "margin": int(rng.integers(0, 12)),
              "max_synth_fraction": float(rng.choice([0.0, 0.02, 0.25, 1.0]))}
    if m.all():
        m[0, 0] = False
    return m, policy


@pytest.mark.parametrize("seed", range(40))
def test_device_census_matches_oracle_on_random_masks(seed):
    mask, policy = _random_mask(seed)
    doc, prov, synth, final = ro.route(mask, **policy)
    result = routing.route_at_floor_mask(mask, routing.RoutingPolicy(**policy))
    assert routing.serialize_routing_json(result) == ro.serialize(doc)
    assert np.array_equal(result.provisional_labels, prov)
    assert np.array_equal(result.synthesis_mask, synth)
    assert np.array_equal(result.final_labels, final)


def test_full_frame_dust_matches_oracle():
    """A full-frame mask (4000 x 5700, 22.8 MP) with thousands of regions."""

    mask = route_cases.dust(21, 4000, 5700, count=6000, rmax=24)
    doc, prov, synth, final = ro.route(mask)
    result = routing.route_at_floor_mask(mask)
    assert routing.serialize_routing_json(result) == ro.serialize(doc)
    assert np.array_equal(result.final_labels, final)
    assert np.array_equal(result.provisional_labels, prov)


# --- primitives -------------------------------------------------------------


def _dev():
    return routing._Device()


@pytest.mark.parametrize("shape, density", [((1, 1), 1.0), ((1, 513), 0.5), ((517, 1), 0.5),
                                            ((255, 257), 0.3), ((500, 700), 0.55),
                                            ((1024, 768), 0.7), ((300, 300), 0.0)])
def test_label8_matches_oracle(shape, density):
    import torch

    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    mask = rng.random(shape) < density
    dev = _dev()
    labels, count = dev.label8(torch.from_numpy(mask.view(np.uint8)).cuda(), *shape)
    expected, expected_count = ro.label8(mask)
    assert count == expected_count
    assert np.array_equal(labels.cpu().numpy(), expected)


@pytest.mark.parametrize("shape, density", [((1, 300), 0.8), ((300, 1), 0.8), ((257, 129), 0.9),
                                            ((600, 450), 0.97), ((64, 64), 0.5)])
def test_chessboard_distance_matches_oracle(shape, density):
    import torch

    rng = np.random.default_rng(shape[0] + 3 * shape[1])
    mask = rng.random(shape) < density
    mask[rng.integers(0, shape[0]), rng.integers(0, shape[1])] = False
    dist = _dev().distance(torch.from_numpy(mask.view(np.uint8)).cuda(), *shape)
    assert np.array_equal(dist.cpu().numpy(), ro.chessboard_distance(mask))


@pytest.mark.parametrize("radius", [0, 1, 3, 17, 5000])
def test_square_dilation_matches_oracle(radius):
    import torch

    rng = np.random.default_rng(radius)
    mask = rng.random((211, 389)) < 0.002
    out = _dev().dilate(torch.from_numpy(mask.view(np.uint8)).cuda(), 211, 389, radius)
    assert np.array_equal(out.cpu().numpy().view(np.bool_), ro.dilate_square(mask, radius))


def test_primitives_reject_bad_arguments():
    lib = _lib.load()
    count = ctypes.c_int64()
    assert lib.fx_label8(None, 4, 4, None, None, None, None, ctypes.byref(count), None) == 1
    assert lib.fx_tile_extract(ctypes.c_void_p(16), 4, 4, 2, 2, 3, 3, 1, ctypes.c_void_p(16),
                               None) == 1  # tile outside the plane: rejected before launch
