"""Many videos of uneven sizes and lengths in one call (gt_batch_videos).

Each video's table must equal what a separate batch() call returns, and the
oracle's, bit for bit: the videos are located one after another and linked
together in one launch of the linker (one CTA per video).
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
