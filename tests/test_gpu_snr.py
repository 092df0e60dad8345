"""snr, minmass_snr and adaptive_background on the GPU against the oracle.

The per-frame image std (the reference's StdArray reduction tree) sets the
candidate threshold (std * snr * rough), the walk's minmass (minmass_snr *
count * std * rough) and the adaptive background passes, which mask the
circles of accepted rows and recompute the std of the masked frame.  Every
column, including linked ids, must equal the oracle's bit for bit.
"""
import numpy as np
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200._params import log_params, trackpy_params
from synth import video
from test_gpu_parity import ALL_TP, assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [
    dict(snr=0.4, minmass=300.0),
    dict(minmass_snr=0.3),
    dict(snr=0.3, minmass_snr=0.4, adaptive_background=1),
    dict(snr=0.3, minmass_snr=0.4, adaptive_background=2),
    dict(snr=0.5, minmass=250.0, adaptive_background=3),
])
@pytest.mark.parametrize("shape", [(128, 128), (64, 128)])
def test_snr_batch_matches_oracle(oracle, kw, shape):
    frames, _ = video(3, shape[0], shape[1], 50, seed=shape[1] + len(kw))
    kw = dict(kw, search_range=5.0)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert len(df) > 20
    assert_same(df, tab, ALL_TP + ["particle"])


def test_snr_float_frames_and_no_doughnut(oracle):
    frames, _ = video(2, 128, 128, 40, seed=61, dtype=np.float32, read_noise=4.0, bg=50.0)
    kw = dict(snr=0.3, minmass_snr=0.3, adaptive_background=2, doughnut_correction=False)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames)
    assert_same(df, tab, ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc"])


def test_snr_with_log_style(oracle):
    frames, _ = video(2, 128, 128, 25, seed=62, dtype=np.float32, read_noise=5.0, bg=50.0, sigma_range=(1.4, 3.0))
    kw = dict(n_radii=6, log_spacing=True, snr=0.2, minmass_snr=0.2, adaptive_background=2)
    df = gt.LoG(frames, 2.0, 5.0, tqdm=False, **kw)
    tab = oracle.batch(log_params(2.0, 5.0, **kw), frames)
    assert_same(df, tab, ["frame", "y", "x", "mass", "r"])


def test_snr_errors():
    frames, _ = video(1, 100, 100, 5, seed=63)
    with pytest.raises(ValueError, match="8\\^k"):
        gt.batch(frames, 9, snr=1.0, tqdm=False)
    ok, _ = video(1, 64, 64, 5, seed=64)
    with pytest.raises(ValueError):
        gt.batch(ok, 9, adaptive_background=0, snr=1.0, tqdm=False)
    with pytest.raises(ValueError):
        gt.batch(ok, 9, adaptive_background=2, tqdm=False)
    # one adaptive pass needs no std: the std buffer stays 0 as in the reference
    gt.batch(ok, 9, adaptive_background=1, minmass=100.0, tqdm=False)


def vignetted(T, H, W, seed):
    frames, _ = video(T, H, W, 40, seed=seed)
    yy, xx = np.mgrid[0:H, 0:W]
    shade = 0.6 + 0.4 * np.exp(-((yy - H * 0.4) ** 2 + (xx - W * 0.6) ** 2) / (0.5 * H * W))
    return np.round(frames * shade).astype(np.uint16)


@pytest.mark.parametrize("kw", [
    dict(correct_illumination=True),
    dict(illumination_sigma=6.0, illumination_correction_per_frame=True),
    dict(illumination_sigma=10.0, snr=0.3, minmass_snr=0.3, adaptive_background=2),
])
def test_illumination_correction_matches_oracle(oracle, kw):
    """Every locate stage sees frame / smoothed profile; the doughnut reads the
    uncorrected frames (the reference's host frames)."""
    frames = vignetted(3, 128, 128, 71)
    kw = dict(kw, minmass=kw.get("minmass", 1.5) if "minmass_snr" not in kw else 0.0, search_range=5.0)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert len(df) > 20
    assert_same(df, tab, ALL_TP + ["particle"])


def test_illumination_with_log(oracle):
    frames = vignetted(2, 96, 128, 72).astype(np.float32)
    kw = dict(n_radii=5, illumination_sigma=8.0)
    df = gt.LoG(frames, 2.0, 4.0, tqdm=False, **kw)
    tab = oracle.batch(log_params(2.0, 4.0, **kw), frames)
    assert_same(df, tab, ["frame", "y", "x", "mass", "r"])
