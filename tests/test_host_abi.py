"""Host logic and the C-ABI surface (no GPU needed).

* the library loads and exports every entry point include/fauxice_b200.h
  declares, with matching struct layouts;
* the host-side prelude entry points (prepass reduction, stage table) match
  the reference / oracle bit for bit;
* profile validation fails closed with the reference's messages;
* the backend refuses to run (fail closed) when no device is present.
"""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

import cases
from _helpers import make_job, sha
from fauxice_b200 import _lib, contracts, profile
from fauxice_b200.engine import B200BackendUnavailable, process_b200
from oracle import oracle as ox

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fauxice_b200.h")


def _declared_symbols() -> set[str]:
    text = open(HEADER).read()
    return set(re.findall(r"FX_API\s+[\w\s\*]+?\b(fx_\w+)\s*\(", text))


def test_header_and_binding_agree():
    declared = _declared_symbols()
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _declared_symbols():
        assert hasattr(lib, name), name
    assert lib.fx_version() == 1


def test_struct_layouts_match_the_oracle():
    # fx_params / fx_stage / fx_counters share the oracle's field layout
    assert ctypes.sizeof(_lib.FxParams) == ctypes.sizeof(ox.OxParams)
    assert _lib.STAGE_DTYPE.itemsize == ox.STAGE_DTYPE.itemsize
    # fx_counters carries walk diagnostics beyond the reference's counters
    assert ctypes.sizeof(_lib.FxCounters) == ctypes.sizeof(ox.OxCounters) + 7 * 8


def test_request_entry_points_reject_bad_arguments():
    """fx_cancel, fx_fetch and the two test knobs refuse a null context or an
    out-of-range value without touching a device."""

    lib = _lib.load()
    assert lib.fx_cancel(None, 1) == 1
    assert lib.fx_pass_bytes(None, 16, 16, ctypes.byref(ctypes.c_int64())) == 1
    assert lib.fx_fetch(None, 1, 0, None, None, None, None, None) == 1
    assert lib.fx_set_walk_window(None, 4.5) == 1
    assert lib.fx_set_list_capacity(None, 0) == 1


def test_frame_bytes_estimate_is_sane():
    lib = _lib.load()
    full = lib.fx_frame_bytes(5782, 3946)
    assert 1 << 30 < full < 4 << 30
    assert lib.fx_frame_bytes(0, 8) == -1


@pytest.mark.parametrize("name", ["engine_8x8", "hybrid_256", "self_test_48x64", "tile_edge",
                                  "tile_high_dynamic_range", "gen_9_17x200", "small_crop_512"])
def test_host_prepass_matches_reference(name, golden):
    main, prepass = cases.JOB_CASES[name][0]()
    lut = profile.response_lut()
    payload = (ctypes.c_uint8 * 64)()
    valid, tiles = ctypes.c_int64(), ctypes.c_int64()
    px = np.ascontiguousarray(prepass)
    rc = _lib.load().fx_reduce_prepass(_lib.ptr(px), px.shape[0], px.shape[1], _lib.ptr(lut),
                                      payload, ctypes.byref(valid), ctypes.byref(tiles))
    assert rc == 0
    expected = golden["jobs"][name]
    assert bytes(payload).hex() == expected["prepass_payload"]
    assert valid.value == expected["prepass_valid_pixels"]
    assert tiles.value == expected["prepass_fully_valid_tiles"]


@pytest.mark.parametrize("geometry", cases.PRODUCER_CASES[:4], ids=lambda g: f"{g[0]}x{g[1]}")
def test_host_stage_table_matches_oracle(geometry):
    h, w, seed = geometry
    rows = ox.producer_rows(cases.producer_pixels(h, w, seed))
    expected = ox.stage_table(rows)
    got = np.zeros(h + 6, dtype=_lib.STAGE_DTYPE)
    rc = _lib.load().fx_stage_table(h, _lib.ptr(rows["p1"]), _lib.ptr(rows["p2"]),
                                    _lib.ptr(rows["mean_vis"]), _lib.ptr(rows["mean_ir"]),
                                    ctypes.c_float(1.0), _lib.ptr(got))
    assert rc == 0
    assert got.tobytes() == expected.tobytes()


def test_tables_reproduce_pinned_digests():
    assert profile.response_lut().dtype == np.float32
    high, low = profile.factor_tables()
    assert high.shape == low.shape == (256,)
    low_b, high_b = profile.dither_bounds(profile.response_lut())
    assert np.float32(low_b) == profile.response_lut()[655]
    assert np.float32(high_b) == profile.response_lut()[64879]


def test_profile_parameters_match_oracle_profile():
    c = profile.DEFAULT_PROFILE.hot_path_parameters().to_c()
    o = ox.Params().to_c(ox.response_lut())
    assert bytes(c) == bytes(o)


@pytest.mark.parametrize(
    "field, value, message",
    [
        ("selector", 7, "unsupported selector 7"),
        ("resolution_metric", 500, "unsupported resolution metric 500"),
        ("bit_depth", 8, "unsupported bit depth 8"),
        ("focus_exposure_locked", False, "main capture must retain prepass focus and exposure"),
    ],
)
def test_validation_fails_closed_like_the_reference(field, value, message):
    main, prepass = cases.engine_8x8()
    job = make_job(main, prepass)
    bad = contracts.ProcessingJob(**{**job.__dict__, field: value})
    with pytest.raises(ValueError, match=re.escape(message)):
        profile.DEFAULT_PROFILE.validate_job(bad)


def test_validation_rejects_small_frames_and_non_jobs():
    with pytest.raises(TypeError, match="processing requires a ProcessingJob"):
        profile.DEFAULT_PROFILE.validate_job(object())
    main, prepass = cases.engine_8x8()
    with pytest.raises(ValueError, match="at least 5 rows by 8 columns"):
        profile.DEFAULT_PROFILE.validate_job(make_job(main[:4], prepass))


def test_reference_jobs_are_accepted(golden):
    """A job built with the reference's own contract classes validates."""

    reference = pytest.importorskip("portable_digital_ice")
    main, prepass = cases.engine_8x8()
    job = reference.ProcessingJob(
        acquisition=reference.DualRGBIAcquisition(
            prepass=reference.RGBI16Frame(prepass, reference.AcquisitionEpoch.PREPASS, 285, "p"),
            main=reference.RGBI16Frame(main, reference.AcquisitionEpoch.MAIN, 4000, "m"),
            same_frame_id="x"),
        scanner_model=reference.ScannerModel.NIKON_SUPER_COOLSCAN_5000_ED,
        mode=reference.ProcessingMode.NORMAL, selector=8, resolution_metric=4000, bit_depth=16,
        focus_exposure_locked=True)
    profile.DEFAULT_PROFILE.validate_job(job)


def _gpu_present() -> bool:
    try:
        return _lib.device_check(0)[0] == 0
    except OSError:
        return False


@pytest.mark.skipif(_gpu_present(), reason="a usable GPU is present")
def test_backend_fails_closed_without_a_device():
    main, prepass = cases.engine_8x8()
    output = np.full((8, 8, 3), 4321, np.uint16)
    with pytest.raises(B200BackendUnavailable):
        process_b200(make_job(main, prepass), output_rgb16=output)
    assert np.all(output == 4321)


def test_synthetic_generator_is_deterministic():
    a = cases.generated(11, 40, 50)[0]
    b = cases.generated(11, 40, 50)[0]
    assert sha(a) == sha(b)
    assert a.dtype == np.uint16 and a.shape == (40, 50, 4)
