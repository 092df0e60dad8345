"""Many videos of uneven sizes and lengths in one call (gt_batch_videos).

Each video's table must equal what a separate batch() call returns, and the
oracle's, bit for bit: the videos are located together in ragged waves (one
launch per stage over frames of every size, a replayed CUDA graph, autotuned
wave shapes) or video by video, and linked together in one launch of the
linker (one CTA per video).
"""
import numpy as np
import pandas as pd
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200._params import trackpy_params
from synth import video
from test_gpu_parity import ALL_TP, assert_same

pytestmark = pytest.mark.gpu


def ragged(seed):
    rng = np.random.default_rng(seed)
    vids = []
    for k in range(7):
        H = int(rng.choice([48, 64, 96, 130]))
        W = int(rng.choice([56, 64, 100, 128]))
        T = int(rng.integers(3, 25))
        n = int(max(2, H * W * rng.uniform(1e-3, 3e-3)))
        v, _ = video(T, H, W, n, seed=seed * 100 + k, D=rng.uniform(0.2, 2.0), turnover=0.05)
        vids.append(v)
    return vids


@pytest.mark.parametrize("memory", [0, 2])
def test_batch_videos_equals_separate_calls_and_oracle(oracle, memory):
    vids = ragged(5 + memory)
    kw = dict(minmass=250.0, search_range=5.0, memory=memory)
    outs = gt.batch_videos(vids, 9, **kw)
    assert len(outs) == len(vids)
    for v, df in zip(vids, outs):
        one = gt.batch(v, 9, tqdm=False, **kw)
        pd.testing.assert_frame_equal(df, one)
        tab = oracle.batch(trackpy_params(9, **kw), v.astype(np.float32))
        assert_same(df, tab, ALL_TP + ["particle", "duration"])


def test_batch_videos_without_linking_and_mixed_dtypes():
    vids = ragged(9)
    vids[1] = vids[1].astype(np.float32)
    outs = gt.batch_videos(vids, 9, minmass=250.0)
    for v, df in zip(vids, outs):
        pd.testing.assert_frame_equal(df, gt.batch(v.astype(np.float32), 9, minmass=250.0, tqdm=False))
        assert "particle" not in df.columns
    assert gt.batch_videos([], 9) == []


# ---------------------------------------------------------------- ragged waves
def _hook(name, *argtypes):
    import ctypes

    from gpu_tracking_b200 import _ffi
    f = getattr(_ffi.lib(), name)
    f.argtypes = [ctypes.c_void_p] + list(argtypes)
    f.restype = ctypes.c_int32
    return f


def _set_ragged(mode):
    import ctypes

    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    ctx.check(_hook("gt__set_ragged", ctypes.c_int32)(ctx.handle, mode))


def _ragged_shape():
    import ctypes

    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    seg, budget = ctypes.c_int32(), ctypes.c_int64()
    ctx.check(_hook("gt__ragged_shape", ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64))(
        ctx.handle, ctypes.byref(seg), ctypes.byref(budget)))
    return seg.value, budget.value


def uneven(seed, n=9):
    """Videos whose frames span several strips and segments and end
    mid-tile: sides from 37 to 1100 px, 2 to 14 frames."""
    rng = np.random.default_rng(seed)
    sides = [37, 64, 130, 257, 300, 512, 640, 1100]
    vids = []
    for k in range(n):
        H, W = int(rng.choice(sides)), int(rng.choice(sides))
        T = int(rng.integers(2, 15))
        spots = int(max(3, H * W * rng.uniform(2e-4, 2e-3)))
        v, _ = video(T, H, W, spots, seed=seed * 1000 + k, D=rng.uniform(0.2, 2.0), turnover=0.05)
        vids.append(v)
    return vids


def test_ragged_waves_device_videos_equal_separate_calls(oracle):
    """Device-resident u16 videos, the headline parameter set: every wave
    shape of the autotuner is used (one after another, on waves of one or a
    few frames), the captured stage graph is replayed for every wave, and
    each video's table still equals its own batch() call and the oracle."""
    torch = pytest.importorskip("torch")
    vids = uneven(21)
    dev = [torch.from_numpy(np.ascontiguousarray(v.astype(np.uint16))).cuda() for v in vids]
    kw = dict(minmass=220.0, separation=12, search_range=7.0, memory=3)
    _set_ragged(2)
    try:
        outs = gt.batch_videos(dev, 11, **kw)
        seg, budget = _ragged_shape()
    finally:
        _set_ragged(1)
    assert seg in (128, 256, 512) and budget > 0
    for v, d, df in zip(vids, dev, outs):
        pd.testing.assert_frame_equal(df, gt.batch(d, 11, tqdm=False, **kw))
    for k in (0, 3, 7):
        tab = oracle.batch(trackpy_params(11, **kw), vids[k].astype(np.float32))
        assert_same(outs[k], tab, ALL_TP + ["particle", "duration"])


@pytest.mark.parametrize("dtype", [np.uint8, np.float32])
def test_ragged_waves_host_videos_equal_video_by_video(dtype):
    """Host videos (staged into double-buffered device memory per wave), u8
    and f32 frames: the ragged waves give the same tables as locating video
    by video."""
    vids = [np.clip(v, 0, 255).astype(dtype) if dtype == np.uint8 else v.astype(dtype) for v in uneven(33, n=7)]
    kw = dict(minmass=120.0, search_range=5.0, memory=1)
    _set_ragged(2)
    try:
        waves = gt.batch_videos(vids, 9, **kw)
    finally:
        _set_ragged(0)
    try:
        one_by_one = gt.batch_videos(vids, 9, **kw)
    finally:
        _set_ragged(1)
    for a, b in zip(waves, one_by_one):
        pd.testing.assert_frame_equal(a, b)
    assert sum(len(a) for a in waves) > 0
