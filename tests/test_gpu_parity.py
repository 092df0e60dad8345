"""CUDA engine vs the CPU oracle, through the C ABI, on seeded synthetic videos.

Integer and index work (candidates, counts, particle ids, durations) must be
identical; the float columns are bit-identical too, because the kernels
evaluate the same IEEE binary32 operation sequence as the oracle (fused
multiply-adds only where the shaders accumulate `acc += a * b`, tables for the
transcendental functions).  FLOAT_TOL is the tolerance written into the
comparison for the float columns; it is zero ULP.
"""
import numpy as np
import pandas as pd
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200._params import COLUMN_INDEX, log_params, trackpy_params
from synth import video

pytestmark = pytest.mark.gpu

FLOAT_TOL_ULP = 0


def oracle_frame(oracle, params, frames, **kw):
    tab = oracle.batch(params, frames.astype(np.float32), **kw)
    return tab


def assert_same(df, tab, cols):
    assert len(df) == len(tab), "row count %d != oracle %d" % (len(df), len(tab))
    for name in cols:
        got = df[name].to_numpy()
        want = tab[:, COLUMN_INDEX[name]]
        if name in ("frame", "particle", "duration"):
            assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), name
        else:
            g32 = got.astype(np.float32)
            w32 = want.astype(np.float32)
            same = (g32.view(np.uint32) == w32.view(np.uint32)) | (np.isnan(g32) & np.isnan(w32))
            if FLOAT_TOL_ULP:
                diff = np.abs(g32.view(np.int32).astype(np.int64) - w32.view(np.int32).astype(np.int64))
                same |= diff <= FLOAT_TOL_ULP
            bad = np.flatnonzero(~same)
            assert bad.size == 0, "%s differs at %d rows, first %s: gpu %r oracle %r" % (
                name, bad.size, bad[:5], g32[bad[:5]], w32[bad[:5]])


ALL_TP = ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc", "raw_mass", "raw_bg_median",
          "raw_mass_corrected"]


@pytest.mark.parametrize("shape,n,diam,minmass,sep", [
    ((128, 160), 40, 9, 500.0, 9),
    ((96, 96), 25, 11, 300.0, None),
    ((17, 23), 2, 5, 50.0, None),
    ((200, 64), 30, 7, 200.0, 4),
])
def test_locate_matches_oracle(oracle, shape, n, diam, minmass, sep):
    frames, _ = video(3, shape[0], shape[1], n, seed=shape[0] + n)
    kw = dict(minmass=minmass)
    if sep is not None:
        kw["separation"] = sep
    df = gt.batch(frames, diam, tqdm=False, **kw)
    p = trackpy_params(diam, **kw)
    tab = oracle.batch(p, frames.astype(np.float32))
    assert_same(df, tab, ALL_TP)


def test_locate_without_filter_and_doughnut(oracle):
    frames, _ = video(2, 80, 90, 30, seed=3)
    kw = dict(minmass=100.0, filter_close=False, doughnut_correction=False, characterize=False)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert list(df.columns) == ["frame", "y", "x", "mass"]
    assert_same(df, tab, ["frame", "y", "x", "mass"])


def test_minmass_zero_and_no_truncation(oracle):
    frames, _ = video(2, 48, 64, 10, seed=4)
    kw = dict(minmass=0.0, truncate_preprocessed=False)
    df = gt.batch(frames, 7, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(7, **kw), frames.astype(np.float32))
    assert_same(df, tab, ALL_TP)


def test_float_and_u8_inputs(oracle):
    frames, _ = video(2, 64, 72, 15, seed=5, dtype=np.float32, read_noise=4.0, bg=50.0)
    df = gt.batch(frames, 9, minmass=200.0, tqdm=False)
    tab = oracle.batch(trackpy_params(9, minmass=200.0), frames)
    assert_same(df, tab, ALL_TP)
    f8, _ = video(2, 64, 72, 15, seed=6, dtype=np.uint8, bg=20.0, amp_mu=np.log(100.0))
    df8 = gt.batch(f8, 9, minmass=50.0, tqdm=False)
    tab8 = oracle.batch(trackpy_params(9, minmass=50.0), f8.astype(np.float32))
    assert_same(df8, tab8, ALL_TP)


def test_link_in_batch_matches_oracle(oracle):
    frames, _ = video(12, 128, 128, 40, seed=7, D=1.0, turnover=0.05)
    kw = dict(minmass=500.0, search_range=5.0, memory=0)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert_same(df, tab, ALL_TP + ["particle", "duration"])
    kw["memory"] = 3
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert_same(df, tab, ALL_TP + ["particle", "duration"])


def test_frames_selection_and_reset_points(oracle):
    frames, _ = video(8, 64, 64, 15, seed=8, D=0.5)
    keys = [0, 1, 2, 5, 6, 7]
    kw = dict(minmass=300.0, search_range=4.0, memory=1)
    df = gt.batch(frames, 9, frames=keys, linker_reset_points=[5], tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames[keys].astype(np.float32), frame_numbers=keys,
                       reset_points=[5])
    assert_same(df, tab, ["frame", "y", "x", "mass", "particle"])


def test_host_and_device_inputs_agree():
    torch = pytest.importorskip("torch")
    frames, _ = video(5, 96, 128, 30, seed=9)
    a = gt.batch(frames, 9, minmass=400.0, search_range=5.0, tqdm=False)
    b = gt.batch(torch.from_numpy(frames.astype(np.int32)).to(torch.uint16).cuda(), 9, minmass=400.0,
                 search_range=5.0, tqdm=False)
    pd.testing.assert_frame_equal(a, b)


@pytest.mark.parametrize("log_spacing,overlap", [(False, 0.0), (True, 0.0), (True, 0.5), (False, 1.0)])
def test_log_matches_oracle(oracle, log_spacing, overlap):
    frames, _ = video(2, 80, 96, 20, seed=10, dtype=np.float32, read_noise=5.0, bg=50.0,
                      sigma_range=(1.4, 4.0))
    kw = dict(n_radii=5, log_spacing=log_spacing, overlap_threshold=overlap, minmass=0.0)
    df = gt.LoG(frames, 2.0, 6.0, tqdm=False, **kw)
    tab = oracle.batch(log_params(2.0, 6.0, **kw), frames)
    assert_same(df, tab, ["frame", "y", "x", "mass", "r", "Rg", "raw", "signal", "ecc", "raw_mass",
                          "raw_bg_median", "raw_mass_corrected"])


def test_characterize_points_matches_oracle(oracle):
    frames, _ = video(4, 64, 80, 12, seed=11)
    rng = np.random.default_rng(1)
    pts = pd.DataFrame({"frame": np.repeat([1, 2, 3], 10).astype(float),
                        "y": rng.uniform(2, 61, 30), "x": rng.uniform(2, 77, 30)})
    df = gt.characterize_points(frames, pts, diameter=9, tqdm=False)
    tab = oracle.characterize_points(trackpy_params(9), frames.astype(np.float32),
                                     pts[["frame", "y", "x"]].to_numpy(np.float32), True, False)
    assert_same(df, tab, ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc", "raw_mass",
                          "raw_bg_median", "raw_mass_corrected"])
    # without a frame column every frame characterizes every point; r column
    pts2 = pd.DataFrame({"y": [10.0, 30.5, 50.2], "x": [12.0, 40.0, 70.7], "r": [3.0, 4.5, 2.2]})
    df2 = gt.characterize_points(frames, pts2, tqdm=False)
    tab2 = oracle.characterize_points(trackpy_params(2 * int(4.5 + 0.5) + 1), frames.astype(np.float32),
                                      pts2.to_numpy(np.float32), False, True)
    assert_same(df2, tab2, ["frame", "y", "x", "mass", "r", "Rg", "raw", "signal", "ecc"])


def random_detections(seed, T=30, n=60, R=4.0, turnover=0.1, size=100.0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, size, (n, 2))
    rows = []
    for t in range(T):
        keep = rng.random(n) > 0.05
        for k in np.flatnonzero(keep):
            rows.append((t, pos[k, 0], pos[k, 1]))
        pos = pos + rng.normal(0, R / 3, pos.shape)
        dead = rng.random(n) < turnover
        pos[dead] = rng.uniform(0, size, (dead.sum(), 2))
    return np.array(rows, np.float32)


@pytest.mark.parametrize("memory", [0, 1, 3])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_link_matches_oracle(oracle, memory, seed):
    rows = random_detections(seed)
    ids = gt.link(rows, 4.0, memory)
    want = oracle.link(rows, 4.0, memory)
    assert np.array_equal(ids, want)


@pytest.mark.parametrize("n,size,R", [(80, 60.0, 5.0), (100, 80.0, 5.0), (120, 80.0, 4.0)])
def test_link_dense_subnets(oracle, n, size, R):
    # crowded: many multi-source multi-destination subnets
    rows = random_detections(5, T=10, n=n, R=R, size=size)
    ids = gt.link(rows, R, 1)
    assert np.array_equal(ids, oracle.link(rows, R, 1))


@pytest.mark.parametrize("n", [3000, 5000])
def test_link_large_frames(oracle, n):
    """Frames of 3000 detections keep the linker's per-frame working arrays in
    shared memory only with 32-bit list offsets; frames of 5000 exceed it and
    use the global scratch.  Both give the oracle's ids."""
    rows = random_detections(7, T=6, n=n, R=5.0, size=1500.0)
    ids = gt.link(rows, 5.0, 2)
    assert np.array_equal(ids, oracle.link(rows, 5.0, 2))


def test_link_load_guard_agrees_with_oracle(oracle):
    rows = random_detections(5, T=10, n=150, R=6.0, size=60.0)
    with pytest.raises(oracle.OracleError):
        oracle.link(rows, 6.0, 1)
    with pytest.raises(ValueError, match="computational load"):
        gt.link(rows, 6.0, 1)


def test_link_too_dense_raises():
    rng = np.random.default_rng(0)
    n = 72
    rows = np.r_[np.c_[np.zeros(n), rng.uniform(0, 1, (n, 2))], np.c_[np.ones(n), rng.uniform(0, 1, (n, 2))]]
    with pytest.raises(ValueError):
        gt.link(rows.astype(np.float32), 5.0, 0)


def test_link_quirks(oracle):
    rows = np.array([[3, 1, 1], [7, 1.5, 1.0], [7, 10, 10]], np.float32)
    assert np.array_equal(gt.link(rows, 2.0, 0), oracle.link(rows, 2.0, 0))
    with pytest.raises(ValueError):
        gt.link(np.array([[1, 0, 0], [0, 1, 1]], np.float32), 2.0, 0)
    assert len(gt.link(np.zeros((0, 3), np.float32), 2.0, 0)) == 0


def test_connect_matches_oracle(oracle):
    a = random_detections(3, T=8, n=30)
    b = a.copy()
    b[:, 1:] += np.random.default_rng(4).normal(0, 0.3, (len(b), 2)).astype(np.float32)
    b = b[np.random.default_rng(5).random(len(b)) > 0.2]
    r1, r2 = gt.connect(a, b, 1.0, merge=False)
    o1, o2 = oracle.connect(a, b, 1.0)
    assert np.array_equal(r1, o1) and np.array_equal(r2, o2)
    # frames present in only one of the inputs
    c = b[b[:, 0] != 3]
    r1, r2 = gt.connect(a, c, 1.0, merge=False)
    o1, o2 = oracle.connect(a, c, 1.0)
    assert np.array_equal(r1, o1) and np.array_equal(r2, o2)


def test_empty_results_and_columns():
    frames = np.full((2, 40, 40), 100, np.uint16)
    df = gt.batch(frames, 9, minmass=1e9, search_range=3.0, tqdm=False)
    assert len(df) == 0
    assert list(df.columns) == ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc", "raw_mass",
                                "raw_bg_median", "raw_mass_corrected", "particle", "duration"]


def test_mean_from_file(tmp_path):
    frames, _ = video(5, 30, 40, 5, seed=12)
    path = tmp_path / "v.npy"
    np.save(path, frames)
    m = gt.mean_from_file(str(path))
    acc = np.zeros((30, 40), np.float32)
    for f in frames.astype(np.float32):
        acc = acc + f
    assert np.array_equal(m, acc / np.float32(5))


def test_errors():
    with pytest.raises(ValueError):
        gt.batch(np.zeros((0, 10, 10), np.uint16), 5, tqdm=False)
    with pytest.raises(ValueError):
        gt.load("file.avi")
    with pytest.raises(FileNotFoundError):
        gt.load("/nonexistent/file.npy")


@pytest.mark.parametrize("diam,sep", [(9, None), (11, None), (9, 9), (7, None), (5, None), (13, None), (9, 30)])
def test_strip_segments_and_generic_fallback(oracle, diam, sep):
    """Tall frames split into several row segments, widths that are not a
    multiple of the strip width, and a dilation size without a specialised
    kernel (separation 30)."""
    frames, _ = video(2, 1100, 300, 160, seed=diam * 3 + (sep or 0))
    kw = dict(minmass=300.0, doughnut_correction=False)
    if sep is not None:
        kw["separation"] = sep
    df = gt.batch(frames, diam, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(diam, **kw), frames.astype(np.float32))
    assert_same(df, tab, ["frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc"])


@pytest.mark.parametrize("dtype,width", [(np.uint16, 520), (np.uint16, 522), (np.uint8, 520), (np.float32, 520),
                                         (np.uint16, 1030)])
def test_strip_interior_strips_and_pixel_types(oracle, dtype, width):
    """Frames wide enough for interior strips (4-pixel staging loads), a width
    that is not a multiple of 4 (per-pixel staging), and every pixel type."""
    kw = dict(bg=40.0, amp_mu=np.log(120.0)) if dtype == np.uint8 else {}
    if dtype == np.float32:
        kw = dict(read_noise=4.0, bg=50.0)
    frames, _ = video(2, 260, width, 150, seed=width + 7, dtype=dtype, **kw)
    mm = 60.0 if dtype == np.uint8 else 300.0
    df = gt.batch(frames, 11, minmass=mm, tqdm=False)
    tab = oracle.batch(trackpy_params(11, minmass=mm), frames.astype(np.float32))
    assert_same(df, tab, ALL_TP)


def plateau_video():
    """Noise-free background with a few spots: the processed image is exactly
    0 on wide plateaus, whose pixels are all local maxima."""
    rng = np.random.default_rng(3)
    fr = np.full((2, 96, 100), 100.0)
    yy, xx = np.mgrid[0:96, 0:100]
    for t in range(2):
        for _ in range(6):
            y, x = rng.uniform(10, 86), rng.uniform(10, 90)
            fr[t] += 600 * np.exp(-((yy - y) ** 2 + (xx - x) ** 2) / (2 * 1.5 ** 2))
    return np.round(fr).astype(np.uint16)


@pytest.mark.parametrize("minmass", [0.0, 100.0])
def test_zero_plateau_candidates(oracle, minmass):
    """minmass = 0 keeps the walks of zero-valued local maxima (mass 0 >= 0),
    so none may be left out; with minmass > 0 they are all rejected and the
    kernels skip them."""
    frames = plateau_video()
    kw = dict(minmass=minmass, separation=14)
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    if minmass == 0.0:
        assert (df["mass"] == 0).sum() > 1000
    assert_same(df, tab, ALL_TP)


@pytest.mark.parametrize("bg_radius,gap_radius", [(9.0, None), (14.0, 2.0), (20.0, None)])
def test_doughnut_annulus_sizes(oracle, bg_radius, gap_radius):
    """Doughnut correction with annuli small and large enough for both median
    paths (register-resident and histogram radix select), spots at the edges."""
    frames, _ = video(2, 120, 136, 35, seed=int(bg_radius) + 40, margin=1.0)
    kw = dict(minmass=300.0, bg_radius=bg_radius)
    if gap_radius is not None:
        kw["gap_radius"] = gap_radius
    df = gt.batch(frames, 9, tqdm=False, **kw)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert_same(df, tab, ALL_TP)
