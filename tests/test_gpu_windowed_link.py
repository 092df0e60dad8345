"""Linking inside gt_batch runs window by window beside the locate kernels.

Each super-chunk of located frames (128 frames for small frames) is linked on
its own stream while the next one is located; the linker's state carries over
between windows.  These videos are long enough to span several windows, and
the ids and durations must equal the oracle's exactly — across window
boundaries, with memory, with linker resets and frame-number gaps on and next
to a boundary, and when the window buffers are forced too small so that the
call falls back to the whole-video linker.
"""
import ctypes

import numpy as np
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200._params import trackpy_params
from synth import video
from test_gpu_parity import ALL_TP, assert_same

pytestmark = pytest.mark.gpu

LINK_COLS = ALL_TP + ["particle", "duration"]


@pytest.fixture(scope="module")
def long_video():
    frames, _ = video(300, 64, 64, 14, seed=21, D=0.6, turnover=0.03)
    return frames


@pytest.mark.parametrize("memory,radius", [(0, 4.0), (3, 4.0), (1, 6.0)])
def test_windows_match_oracle(oracle, long_video, memory, radius):
    kw = dict(minmass=300.0, search_range=radius, memory=memory)
    df = gt.batch(long_video, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), long_video.astype(np.float32))
    assert df["frame"].max() == 299
    assert_same(df, tab, LINK_COLS)


KEYS = [k for k in range(300) if k not in (126, 200, 201)]


def test_resets_and_gaps_at_window_boundaries(oracle, long_video):
    resets = [60, 127, 128, 129]
    kw = dict(minmass=300.0, search_range=4.0, memory=2)
    df = gt.batch(long_video, 9, frames=KEYS, linker_reset_points=resets, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), long_video[KEYS].astype(np.float32), frame_numbers=KEYS,
                       reset_points=resets)
    assert_same(df, tab, LINK_COLS)


def test_reset_leaving_ids_without_duration_raises_like_oracle(oracle, long_video):
    # the last segment (frames 250..299) hands out fewer ids than earlier ones;
    # the reference's duration lookup panics on the larger ids
    from oracle.loader import OracleError
    resets = [127, 128, 129, 250]
    kw = dict(minmass=300.0, search_range=4.0, memory=2)
    with pytest.raises(OracleError):
        oracle.batch(trackpy_params(9, **kw), long_video[KEYS].astype(np.float32), frame_numbers=KEYS,
                     reset_points=resets)
    from gpu_tracking_b200._ffi import GpuTrackingError
    with pytest.raises(GpuTrackingError, match="no duration entry"):
        gt.batch(long_video, 9, frames=KEYS, linker_reset_points=resets, tqdm=False, **kw)


@pytest.mark.parametrize("list_entries,edges", [(64, 1 << 20), (1 << 22, 4)])
def test_fallback_to_whole_video_linker(oracle, long_video, list_entries, edges):
    from gpu_tracking_b200 import _ffi
    L = _ffi.lib()
    L.gt__set_link_window_caps.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]
    L.gt__set_link_window_caps.restype = ctypes.c_int32
    ctx = _ffi.context(0)
    kw = dict(minmass=300.0, search_range=4.0, memory=3)
    tab = oracle.batch(trackpy_params(9, **kw), long_video.astype(np.float32))
    try:
        ctx.check(L.gt__set_link_window_caps(ctx.handle, list_entries, edges))
        df = gt.batch(long_video, 9, tqdm=False, **kw)
        assert_same(df, tab, LINK_COLS)
    finally:
        ctx.check(L.gt__set_link_window_caps(ctx.handle, 0, 0))
    df = gt.batch(long_video, 9, tqdm=False, **kw)
    assert_same(df, tab, LINK_COLS)
