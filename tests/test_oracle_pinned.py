"""The oracle against the reference's own WGSL shaders executed on the CPU.

oracle/wgsl2cpp.py translates the reference's shader sources into C++
(oracle/_ref/, built from the reference checkout); the restatement in
oracle/gt_oracle.cpp must agree with them bit for bit on every stage.
"""
import numpy as np
import pytest

from gpu_tracking_b200._params import log_params, trackpy_params
from synth import video

pytestmark = pytest.mark.skipif(
    not __import__("oracle.loader", fromlist=["x"]).ref_available(),
    reason="reference translation not built (needs the reference checkout: make -C oracle ref)")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


CASES = [
    dict(diameter=9, minmass=500, separation=9),
    dict(diameter=11, minmass=300),
    dict(diameter=7, minmass=0, truncate_preprocessed=False),
    dict(diameter=9, minmass=100, smoothing_size=13, noise_size=1.3, shift_threshold=0.55),
    dict(diameter=10, minmass=200, separation=4, max_iterations=3),
]


@pytest.mark.parametrize("kw", CASES)
@pytest.mark.parametrize("shape", [(64, 96), (37, 53)])
def test_trackpy_stages_bit_exact(oracle, kw, shape):
    kw = dict(kw)
    seed = (shape[0] * 31 + kw["diameter"] * 7 + int(kw["minmass"])) % 1000
    frames, _ = video(2, shape[0], shape[1], 12, seed=seed)
    p = trackpy_params(kw.pop("diameter"), **kw)
    for f in frames.astype(np.float32):
        a, b = oracle.preprocess(p, f), oracle.ref_preprocess(p, f)
        assert np.array_equal(bits(a), bits(b))
        ca, cb = oracle.candidates(p, a), oracle.ref_candidates(p, b)
        assert np.array_equal(ca, cb)
        rows, keep = oracle.walk(p, a, f, ca)
        rr = oracle.ref_walk(p, b, f, cb, characterize=True)
        assert np.array_equal(bits(rows[keep]), bits(rr))


def test_characterize_points_bit_exact(oracle):
    frames, _ = video(1, 60, 70, 10, seed=5)
    f = frames[0].astype(np.float32)
    p = trackpy_params(9)
    rng = np.random.default_rng(0)
    pts = np.c_[rng.uniform(0, 59, 40), rng.uniform(0, 69, 40)].astype(np.float32)
    pts[:3] = [[10.5, 20.5], [11.5, 21.5], [0.0, 0.0]]   # half-way rounding and a corner
    proc = oracle.preprocess(p, f)
    rr = oracle.ref_characterize_points(p, proc, f, pts)
    tab = oracle.characterize_points(p, frames.astype(np.float32), pts, False, False)
    # columns: mass, Rg, raw, signal, ecc  vs ResultRow fields 2, 5, 6, 7, 8
    assert np.array_equal(bits(tab[:, 3]), bits(rr[:, 2]))
    for col, field in ((5, 5), (6, 6), (7, 7), (8, 8)):
        assert np.array_equal(bits(tab[:, col]), bits(rr[:, field]))


@pytest.mark.parametrize("log_spacing", [False, True])
def test_log_planes_and_maxima_bit_exact(oracle, log_spacing):
    frames, _ = video(1, 48, 56, 10, seed=7, dtype=np.float32, read_noise=5.0, bg=50.0)
    f = frames[0]
    p = log_params(2.0, 6.0, n_radii=4, log_spacing=log_spacing)
    planes, radii = oracle.log_planes(p, f)
    proc = oracle.preprocess(p, f)
    for i, r in enumerate(radii):
        ref = oracle.ref_laplace(p, f, np.float32(r) / np.sqrt(np.float32(2.0)))
        assert np.array_equal(bits(planes[i]), bits(ref))
    n = len(radii)
    for i in range(n):
        edge = -1 if i == 0 else (1 if i == n - 1 else 0)
        bottom = planes[i - 1] if i > 0 else np.zeros_like(f)
        top = planes[i + 1] if i < n - 1 else np.zeros_like(f)
        cands = oracle.ref_logspace_max(p, bottom, planes[i], top, proc, edge, radii[i])
        rows = oracle.ref_walk(p, proc, f, cands, r=float(radii[i]), characterize=False)
        mine, keep = oracle.walk(p, proc, f, cands, r=float(radii[i]))
        assert np.array_equal(bits(mine[keep][:, :5]), bits(rows[:, :5]))


def test_full_batch_counts_match_reference_stages(oracle):
    """Per-frame walk output of the reference equals the oracle's pre-filter rows."""
    frames, _ = video(3, 80, 80, 20, seed=11)
    p = trackpy_params(9, minmass=400, separation=9, filter_close=False, doughnut_correction=False)
    tab = oracle.batch(p, frames.astype(np.float32))
    for t, f in enumerate(frames.astype(np.float32)):
        proc = oracle.ref_preprocess(p, f)
        rr = oracle.ref_walk(p, proc, f, oracle.ref_candidates(p, proc))
        mine = tab[tab[:, 0] == t]
        assert len(mine) == len(rr)
        assert np.array_equal(bits(mine[:, 1]), bits(rr[:, 0]))
        assert np.array_equal(bits(mine[:, 2]), bits(rr[:, 1]))
        assert np.array_equal(bits(mine[:, 3]), bits(rr[:, 2]))
