"""snr / minmass_snr / adaptive_background: the oracle against the reference's
own shaders (sum_image_outplace, sum_image_inplace, last_reduction,
std_image, extract_max, walk, adaptive_filter) executed on the CPU.

The frame std is the reference's fixed tree of 8-way sums; it is pinned bit
for bit, with masked pixels (the 0xFFFFFFFF pattern the adaptive filter
writes) and a decremented divisor.  Frame sizes are ones where every level of
that tree divides by 8 (the only sizes whose result does not depend on what
earlier passes left in the reference's shared temp buffer).
"""
import numpy as np
import pytest

from gpu_tracking_b200._params import trackpy_params
from synth import video

loader = __import__("oracle.loader", fromlist=["x"])
pytestmark = pytest.mark.skipif(not loader.ref_available(),
                                reason="reference translation not built (make -C oracle ref)")

MASK = np.uint32(0xFFFFFFFF).view(np.float32)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("shape", [(64, 64), (32, 64), (128, 256), (64, 96)])
@pytest.mark.parametrize("masked", [0.0, 0.15])
def test_frame_std_bit_exact(oracle, shape, masked):
    rng = np.random.default_rng(shape[0] + int(masked * 100))
    f = rng.poisson(100.0, shape).astype(np.float32) + rng.normal(0, 3, shape).astype(np.float32)
    m = rng.random(shape) < masked
    f[m] = MASK
    div = f.size - int(m.sum())
    a = oracle.frame_std(f, div)
    b = oracle.ref_frame_std(f, div)
    assert bits(a) == bits(b)
    assert 2.0 < float(a) < 20.0


def test_frame_std_rejects_sizes_with_inexact_reduction(oracle):
    f = np.ones((37, 53), np.float32)
    with pytest.raises(loader.OracleError):
        oracle.frame_std(f)


@pytest.mark.parametrize("kw", [dict(snr=1.5, minmass=300.0), dict(minmass_snr=2.0), dict(snr=0.8, minmass_snr=1.2),
                                dict(snr=1.0, minmass_snr=1.0, adaptive_background=2)])
def test_snr_candidates_and_walk_bit_exact(oracle, kw):
    frames, _ = video(1, 64, 96, 14, seed=41)
    f = frames[0].astype(np.float32)
    p = trackpy_params(9, **kw)
    sd = oracle.frame_std(f)
    assert bits(sd) == bits(oracle.ref_frame_std(f))
    proc = oracle.preprocess(p, f)
    ca, cb = oracle.candidates(p, proc, float(sd)), oracle.ref_candidates(p, proc, float(sd))
    assert np.array_equal(ca, cb)
    assert len(ca) < len(oracle.candidates(p, proc, 0.0)) or "snr" not in kw
    rows, keep = oracle.walk(p, proc, f, ca, pic_std=float(sd))
    rr = oracle.ref_walk(p, proc, f, cb, characterize=True, pic_std=float(sd))
    assert np.array_equal(bits(rows[keep]), bits(rr))


@pytest.mark.parametrize("n_iter", [1, 2, 3])
@pytest.mark.parametrize("kw", [dict(snr=0.3, minmass_snr=0.4), dict(snr=0.5, minmass=250.0)])
def test_adaptive_filter_bit_exact(oracle, n_iter, kw):
    frames, _ = video(1, 64, 128, 60, seed=43 + n_iter)
    f = frames[0].astype(np.float32)
    p = trackpy_params(9, adaptive_background=n_iter, **kw)
    sd = float(oracle.frame_std(f))
    proc = oracle.preprocess(p, f)
    cands = oracle.candidates(p, proc, sd)
    rows, keep = oracle.walk(p, proc, f, cands, pic_std=sd)
    walked = rows[keep]
    assert len(walked) > 10
    mine = oracle.adaptive(p, f, walked, n_iter, sd)
    ref = oracle.ref_adaptive(p, f, walked, n_iter, sd)
    assert len(mine) == len(ref)
    order = lambda r: np.lexsort((bits(r[:, 1]), bits(r[:, 0])))  # noqa: E731
    assert np.array_equal(bits(mine[order(mine)]), bits(ref[order(ref)]))
    if n_iter > 1:
        # later passes see a masked frame: fewer or equal acceptances than one pass would give
        assert len(mine) >= len(oracle.adaptive(p, f, walked, 1, sd))


@pytest.mark.parametrize("sigma,shape", [(3.0, (40, 56)), (7.5, (64, 48)), (30.0, (33, 70))])
def test_illumination_profile_and_correction_bit_exact(oracle, sigma, shape):
    """smooth_mean_frame.wgsl (two separable passes) and correct_illumination.wgsl."""
    rng = np.random.default_rng(int(sigma * 10))
    yy, xx = np.mgrid[0:shape[0], 0:shape[1]]
    prof = (100 + 40 * np.exp(-((yy - shape[0] / 3) ** 2 + (xx - shape[1] / 2) ** 2) / 400.0)).astype(np.float32)
    frame = (prof * rng.uniform(0.5, 2.0, shape)).astype(np.float32)
    p = trackpy_params(9, illumination_sigma=sigma)
    smooth, corrected = oracle.ref_illumination(p, prof, sigma, frame)
    mine = oracle.smooth_profile(prof, sigma)
    assert np.array_equal(bits(mine), bits(smooth))
    assert np.array_equal(bits(frame / mine), bits(corrected))
