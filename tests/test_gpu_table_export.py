"""gt_table_export: every column of a table of some 400k rows, moved in
one call through the pinned staging lanes (several lanes, several chunks per
lane), equals the single-column getters: int64 columns bit for bit, float
columns as the exact float64 widening of the float32 column."""
import ctypes

import numpy as np
import pytest

from gpu_tracking_b200 import _ffi
from gpu_tracking_b200._params import COLUMN_INDEX, INT_COLUMNS, NUM_COLUMNS, trackpy_params
from gpu_tracking_b200.synth import brownian_video

pytestmark = pytest.mark.gpu

P32 = ctypes.POINTER(ctypes.c_float)
P64 = ctypes.POINTER(ctypes.c_int64)


def run_batch(video, params):
    ctx = _ffi.context(0)
    out = ctypes.c_void_p()
    import torch
    torch.cuda.synchronize()
    T, H, W = video.shape
    ctx.check(_ffi.lib().gt_batch(ctx.handle, ctypes.byref(params), ctypes.c_void_p(video.data_ptr()), 0, T, H, W,
                                  None, None, 0, ctypes.byref(out)))
    return ctx, out


def export(ctx, handle, names, n):
    L = _ffi.lib()
    data = {c: np.full(n, -7, np.int64 if c in INT_COLUMNS else np.float64) for c in names}
    idx = (ctypes.c_int32 * len(names))(*[COLUMN_INDEX[c] for c in names])
    ptrs = (ctypes.c_void_p * len(names))(*[data[c].ctypes.data for c in names])
    return L.gt_table_export(handle, idx, len(names), ptrs), data


def test_export_equals_single_column_getters():
    video = brownian_video(120, 1024, 1024, 8000, seed=4)
    params = trackpy_params(9, minmass=150.0, search_range=5.0, memory=2)
    ctx, handle = run_batch(video, params)
    L = _ffi.lib()
    try:
        n = L.gt_table_nrows(handle)
        assert n > 300_000, n   # two or more lanes of 256k rows; an int64 chunk is 128k rows
        names = [c for c, i in COLUMN_INDEX.items() if i < NUM_COLUMNS and L.gt_table_has_column(handle, i)]
        assert {"frame", "y", "x", "mass", "particle", "duration"} <= set(names)
        st, got = export(ctx, handle, names, n)
        ctx.check(st)
        for c in names:
            if c in INT_COLUMNS:
                want = np.empty(n, np.int64)
                ctx.check(L.gt_table_column_i64(handle, COLUMN_INDEX[c], want.ctypes.data_as(P64)))
                assert np.array_equal(got[c], want), c
            else:
                want = np.empty(n, np.float32)
                ctx.check(L.gt_table_column_f32(handle, COLUMN_INDEX[c], want.ctypes.data_as(P32)))
                assert got[c].dtype == np.float64
                assert np.array_equal(got[c].view(np.uint64), want.astype(np.float64).view(np.uint64)), c
        # a subset in another order
        st, sub = export(ctx, handle, ["x", "frame"], n)
        ctx.check(st)
        assert np.array_equal(sub["x"], got["x"]) and np.array_equal(sub["frame"], got["frame"])
        # a column index outside the table's columns, and a null destination
        buf = np.empty(n, np.float64)
        idx = (ctypes.c_int32 * 1)(NUM_COLUMNS)
        ptrs = (ctypes.c_void_p * 1)(buf.ctypes.data)
        assert L.gt_table_export(handle, idx, 1, ptrs) == 1   # GT_ERR_INVALID_ARGUMENT
        idx = (ctypes.c_int32 * 1)(COLUMN_INDEX["y"])
        ptrs = (ctypes.c_void_p * 1)(None)
        assert L.gt_table_export(handle, idx, 1, ptrs) == 1
    finally:
        L.gt_table_free(handle)


def test_export_of_an_empty_table():
    video = brownian_video(2, 64, 64, 5, seed=1)
    ctx, handle = run_batch(video, trackpy_params(9, minmass=1e9))
    L = _ffi.lib()
    try:
        assert L.gt_table_nrows(handle) == 0
        st, data = export(ctx, handle, ["frame", "y"], 0)
        ctx.check(st)
    finally:
        L.gt_table_free(handle)


def test_device_frames_must_fit_their_allocation():
    """A device pointer whose dtype or shape claims more bytes than its
    allocation holds is rejected before any kernel reads it.  Every call here
    also asks for a diameter the engine refuses (its smoothing window does not
    fit shared memory), so even without the allocation check no kernel would
    read the frames: the message tells which check answered."""
    import torch
    L = _ffi.lib()
    ctx = _ffi.context(0)
    buf = torch.zeros((4, 256, 256), dtype=torch.uint16, device="cuda")
    torch.cuda.synchronize()
    params = trackpy_params(201)
    out = ctypes.c_void_p()

    def call(ptr, dtype, T):
        st = L.gt_batch(ctx.handle, ctypes.byref(params), ctypes.c_void_p(ptr), dtype, T, 256, 256, None, None, 0,
                        ctypes.byref(out))
        msg = L.gt_last_error(ctx.handle)
        return st, (msg.decode() if msg else "")

    # in bounds: the later parameter check answers
    for ptr, dtype, T in ((buf.data_ptr(), 0, 4), (buf[2].data_ptr(), 0, 2), (buf.data_ptr(), 1, 2)):
        st, msg = call(ptr, dtype, T)
        assert st == 1 and "past the end" not in msg, (T, msg)
    # past the end of the allocation (the caching allocator rounds a block up
    # to 2 MiB, so the claims below exceed any block that holds 512 KiB)
    for ptr, dtype, T in ((buf.data_ptr(), 0, 40), (buf[3].data_ptr(), 1, 20)):
        st, msg = call(ptr, dtype, T)
        assert st == 1 and "past the end" in msg, (T, msg)
