"""Parity at the benchmarked configurations, through the public API.

The workload set's configurations, each compared with the CPU oracle on every
output column, the particle ids and the durations — bit for bit (integer
columns identical; float columns identical to zero ULP, NaN equal to NaN):

* the small plain batch in full: 100 frames of 512x512 uint16, 200 spots per
  frame (sigma 1.5 px, lognormal amplitudes around 800, Brownian D 0.5),
  diameter 9, minmass 500, separation 9, search_range 5, memory 0;
* the headline plain batch's exact parameter set on 136 frames of 2048x2048
  uint16 made by the benchmark's own generator (2000 spots per frame, sigma
  1.2-2.5 px, SNR 3-20, D 1.0, 2 % births/deaths): diameter 11, minmass 220,
  separation 12, characterize, doughnut correction, search_range 7, memory 3.
  136 frames are two super-chunks (128 + 8), so the link stream links across
  a window boundary beside locating, as in the timed run; the video goes in
  once from device memory (the HBM-resident path) and once from host memory
  (the end-to-end path);
* the multi-scale LoG configuration on 3 frames of 1024x1024 float32 (1500
  blobs of radius 2-8 px, read noise 5 on a background of 50): min_radius 2,
  max_radius 8, 10 log-spaced radii, minmass 150, characterize, search_range 6.
"""
import numpy as np
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200._params import COLUMN_INDEX, log_params, trackpy_params
from synth import video

pytestmark = pytest.mark.gpu

TP_COLS = ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc", "raw_mass", "raw_bg_median",
           "raw_mass_corrected", "particle", "duration"]


def assert_table_equal(df, tab, cols):
    assert len(df) == len(tab), "row count %d != oracle %d" % (len(df), len(tab))
    assert len(df) > 0
    for name in cols:
        got = df[name].to_numpy()
        want = tab[:, COLUMN_INDEX[name]]
        if name in ("frame", "particle", "duration"):
            g, w = got.astype(np.int64), want.astype(np.int64)
            bad = np.flatnonzero(g != w)
            assert bad.size == 0, "%s differs at %d rows, first %s: gpu %r oracle %r" % (
                name, bad.size, bad[:5], g[bad[:5]], w[bad[:5]])
        else:
            g32, w32 = got.astype(np.float32), want.astype(np.float32)
            same = (g32.view(np.uint32) == w32.view(np.uint32)) | (np.isnan(g32) & np.isnan(w32))
            bad = np.flatnonzero(~same)
            assert bad.size == 0, "%s differs at %d rows, first %s: gpu %r oracle %r" % (
                name, bad.size, bad[:5], g32[bad[:5]], w32[bad[:5]])


def test_small_plain_batch_in_full(oracle):
    frames, _ = video(100, 512, 512, 200, seed=1, sigma=1.5, amp_mu=np.log(800.0), amp_s=0.5, D=0.5)
    kw = dict(minmass=500.0, separation=9, search_range=5.0, memory=0)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert_table_equal(df, tab, TP_COLS)
    assert df["particle"].nunique() < len(df) / 20


def test_headline_parameter_set_136_frames(oracle):
    torch = pytest.importorskip("torch")
    import bench
    dev_frames = bench.make_video(136, 2048, seed=2, device="cuda")
    torch.cuda.synchronize()
    host = dev_frames.cpu().numpy()
    p = bench.params()
    kw = dict(minmass=220.0, separation=12, search_range=7.0, memory=3)
    assert p.separation == 12 and p.memory == 3 and p.doughnut_correction and p.characterize
    tab = oracle.batch(p, host.astype(np.float32))
    assert len(tab) > 136 * 1500
    df_dev = gt.batch(dev_frames, 11, tqdm=False, **kw)
    assert_table_equal(df_dev, tab, TP_COLS)
    del dev_frames
    df_host = gt.batch(host, 11, tqdm=False, **kw)
    assert_table_equal(df_host, tab, TP_COLS)
    # tracks run across the 128-frame link window
    span = df_dev.groupby("particle")["frame"].agg(["min", "max"])
    assert ((span["min"] < 128) & (span["max"] >= 128)).sum() > 1000


def test_log_configuration_1024sq_10_radii(oracle):
    torch = pytest.importorskip("torch")
    from gpu_tracking_b200.synth import blob_video
    dev_frames = blob_video(3, 1024, 1024, 1500, seed=3, device="cuda")
    torch.cuda.synchronize()
    host = dev_frames.cpu().numpy()
    kw = dict(n_radii=10, log_spacing=True, minmass=150.0, search_range=6.0)
    df = gt.LoG(dev_frames, 2.0, 8.0, tqdm=False, **kw)
    tab = oracle.batch(log_params(2.0, 8.0, **kw), host)
    assert_table_equal(df, tab, ["frame", "y", "x", "mass", "r", "Rg", "raw", "signal", "ecc", "raw_mass",
                                 "raw_bg_median", "raw_mass_corrected", "particle", "duration"])
    assert len(np.unique(df["r"].to_numpy())) >= 8
