"""The no-allocation producer entry point against the allocating one.

fx_producer_rows_static keeps its scratch in a fixed device array instead of
a context allocation.  Its per-row records must equal fx_producer_rows' and
its stage table fx_stage_table's, bit for bit, call after call (a previous
call's scratch contents must not leak into the next).  The file name sorts
last so the test also runs after the rest of the GPU suite used the device.
"""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

import cases
from fauxice_b200 import _lib, engine
from fauxice_b200.synthetic import native_frame

pytestmark = pytest.mark.gpu


def _allocating(ctx, px):
    lib = _lib.load()
    h, w = px.shape[:2]
    px = np.ascontiguousarray(px)
    rows = [np.empty(h, np.float32) for _ in range(4)]
    assert lib.fx_producer_rows(ctx.handle, _lib.ptr(px), h, w, *(_lib.ptr(r) for r in rows)) == 0
    stages = np.zeros(h + 6, dtype=_lib.STAGE_DTYPE)
    rc = lib.fx_stage_table(h, *(_lib.ptr(r) for r in rows), ctypes.c_float(1.0),
                            _lib.ptr(stages))
    return np.concatenate(rows), stages, rc


def _static(ctx, px, stream):
    import torch

    lib = _lib.load()
    h, w = px.shape[:2]
    with torch.cuda.stream(stream):
        d_in = torch.from_numpy(np.ascontiguousarray(px).view(np.int16)).to("cuda")
        d_rows = torch.full((4 * h,), float("nan"), dtype=torch.float32, device="cuda")
        d_stages = torch.full(((h + 6) * _lib.STAGE_DTYPE.itemsize,), 0xA5, dtype=torch.uint8,
                              device="cuda")
    rc = lib.fx_producer_rows_static(ctx.handle, ctypes.c_void_p(d_in.data_ptr()), h, w,
                                     ctypes.c_void_p(d_rows.data_ptr()),
                                     ctypes.c_void_p(d_stages.data_ptr()),
                                     ctypes.c_void_p(stream.cuda_stream))
    with torch.cuda.stream(stream):
        rows = d_rows.cpu().numpy()
        stages = d_stages.cpu().numpy().view(_lib.STAGE_DTYPE)
    return rc, rows, stages


def _frames():
    out = [cases.producer_pixels(h, w, seed) for h, w, seed in cases.PRODUCER_CASES[:3]]
    out.append(cases.producer_pixels(517, 611, 5))
    main, _ = native_frame()  # 5782x3946: the largest frame the scratch holds
    out.append(main)
    return out


def test_static_scratch_matches_allocating_entry_point():
    import torch

    ctx = engine.context()
    stream = torch.cuda.Stream()
    frames = _frames()
    # two passes over the frames: every call follows a call on another frame
    for _ in range(2):
        for px in frames:
            rows, stages, rc_table = _allocating(ctx, px)
            rc, got_rows, got_stages = _static(ctx, px, stream)
            assert rc == rc_table
            assert got_rows.tobytes() == rows.astype(np.float32).tobytes()
            assert got_stages.tobytes() == stages.tobytes()


def test_static_scratch_rejects_oversize_frames():
    import torch

    ctx = engine.context()
    lib = _lib.load()
    small = torch.zeros(64, dtype=torch.uint8, device="cuda")
    p = ctypes.c_void_p(small.data_ptr())
    # rejected on the host from the sizes alone, before any device access
    rc = lib.fx_producer_rows_static(ctx.handle, p, 8192, 8192, p, p, None)
    assert rc == 1
    message = ctx._error(ctx.handle)
    assert re.search(r"8192x8192 frame needs \d+ bytes of producer scratch; the static scratch "
                     r"holds 25165568", message), message
