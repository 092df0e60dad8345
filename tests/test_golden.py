"""Golden vectors from the reference's own shaders (tests/golden/make_golden.py:
preprocess_rows/cols, max_rows + extract_max, walk + characterize, translated
from the reference's WGSL and run on the CPU).  They need no reference
checkout, so they pin the oracle and the GPU path on any machine:

* the oracle's restatement reproduces every processed value, candidate and
  walked row bit for bit;
* the engine's table (filter_close and the doughnut off, so that only the
  shader stages shape it) holds the same rows bit for bit.
"""
import os

import numpy as np
import pytest

from gpu_tracking_b200._params import trackpy_params

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "trackpy_ref_64x96.npz")
# the generator's cases (tests/golden/make_golden.py)
CASES = [
    dict(diameter=9, minmass=300.0, separation=9),
    dict(diameter=11, minmass=200.0),
    dict(diameter=7, minmass=0.0, truncate_preprocessed=False),
    dict(diameter=9, snr=1.2, minmass_snr=0.3),
    dict(diameter=9, minmass=0.05, illumination_sigma=4.0, illumination_correction_per_frame=True),
    dict(diameter=9, adaptive_background=2, snr=0.3, minmass_snr=1.0),
]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same_floats(got, want):
    """Bit-identical float32 values; a NaN equals any NaN (the GPU and the
    host write different NaN payloads, e.g. for Rg of a zero-mass row)."""
    g = np.ascontiguousarray(got, np.float32)
    w = np.ascontiguousarray(want, np.float32)
    return bool(np.all((bits(g) == bits(w)) | (np.isnan(g) & np.isnan(w))))


def by_position(rows):
    """Rows ordered by (row, column) bits (the adaptive passes keep a subset in
    their own order)."""
    return rows[np.lexsort((bits(rows[:, 1]), bits(rows[:, 0])))]


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_reproduces_reference_shaders(oracle, golden, case):
    p = trackpy_params(**CASES[case])
    frames = golden["c%d_frames" % case]
    assert len(golden["c%d_t0_rows" % case]) + len(golden["c%d_t1_rows" % case]) > 0
    for t in range(frames.shape[0]):
        f = frames[t].astype(np.float32)
        if CASES[case].get("illumination_correction_per_frame"):
            f = f / oracle.smooth_profile(f, np.float32(CASES[case]["illumination_sigma"]))
        proc = oracle.preprocess(p, f)
        if t == 0:
            assert np.array_equal(bits(proc), bits(golden["c%d_t0_processed" % case]))
        std = golden["c%d_std" % case][t] if ("snr" in CASES[case] or "minmass_snr" in CASES[case]) else 0.0
        cands = oracle.candidates(p, proc, pic_std=std)
        assert np.array_equal(cands, golden["c%d_t%d_candidates" % (case, t)])
        rows, keep = oracle.walk(p, proc, f, cands, pic_std=std)
        rows = rows[keep]
        want = golden["c%d_t%d_rows" % (case, t)]
        if CASES[case].get("adaptive_background"):
            rows = oracle.adaptive(p, f, rows, CASES[case]["adaptive_background"], std)
            rows, want = by_position(rows), by_position(want)
        assert np.array_equal(bits(rows), bits(want))


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_engine_reproduces_reference_shaders(golden, case):
    import gpu_tracking_b200 as gt
    kw = dict(CASES[case])
    diameter = kw.pop("diameter")
    frames = golden["c%d_frames" % case]
    df = gt.batch(frames, diameter, filter_close=False, doughnut_correction=False, characterize=True, tqdm=False,
                  **kw)
    # walked rows: x (row), y (column), mass, r, max, Rg, raw, signal, ecc, count
    cols = [("y", 0), ("x", 1), ("mass", 2), ("Rg", 5), ("raw", 6), ("signal", 7), ("ecc", 8)]
    for t in range(frames.shape[0]):
        want = golden["c%d_t%d_rows" % (case, t)]
        got = df[df["frame"] == t]
        assert len(got) == len(want), (t, len(got), len(want))
        if CASES[case].get("adaptive_background"):
            want = by_position(want)
            got = got.iloc[np.lexsort((bits(got["x"].to_numpy()), bits(got["y"].to_numpy())))]
        for name, field in cols:
            assert same_floats(got[name].to_numpy(), want[:, field]), (t, name)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_frame_std_matches_reference(oracle, golden, case):
    frames = golden["c%d_frames" % case]
    want = golden["c%d_std" % case]
    got = np.array([oracle.frame_std(f.astype(np.float32)) for f in frames], np.float32)
    assert np.array_equal(bits(got), bits(want))


@pytest.fixture(scope="module")
def golden_log():
    with np.load(os.path.join(HERE, "golden", "log_ref_48x56.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("spacing", [0, 1])
def test_oracle_log_matches_reference(oracle, golden_log, spacing):
    """Scale planes of every radius bit for bit, and the walks from the
    reference's scale-space maxima (position, mass, radius, max)."""
    from gpu_tracking_b200._params import log_params
    f = golden_log["frame"]
    p = log_params(2.0, 6.0, n_radii=4, log_spacing=bool(spacing))
    planes, radii = oracle.log_planes(p, f)
    assert np.array_equal(bits(radii), bits(golden_log["s%d_radii" % spacing]))
    assert np.array_equal(bits(planes), bits(golden_log["s%d_planes" % spacing]))
    proc = oracle.preprocess(p, f)
    n_rows = 0
    for i, r in enumerate(radii):
        cands = golden_log["s%d_r%d_candidates" % (spacing, i)]
        want = golden_log["s%d_r%d_rows" % (spacing, i)]
        mine, keep = oracle.walk(p, proc, f, cands, r=float(r))
        assert np.array_equal(bits(mine[keep][:, :5]), bits(want[:, :5])), i
        n_rows += len(want)
    assert n_rows > 0


@pytest.mark.gpu
@pytest.mark.parametrize("spacing", [0, 1])
def test_engine_log_matches_reference(golden_log, spacing):
    """The engine's LoG detections (no pruning, no characterization) are the
    walks from the reference's scale-space maxima: position, mass and radius
    bit for bit."""
    import gpu_tracking_b200 as gt
    f = golden_log["frame"]
    df = gt.LoG(f[None], 2.0, 6.0, n_radii=4, log_spacing=bool(spacing), overlap_threshold=1.0,
                characterize=False, doughnut_correction=False, tqdm=False)
    radii = golden_log["s%d_radii" % spacing]
    want = np.concatenate([golden_log["s%d_r%d_rows" % (spacing, i)] for i in range(len(radii))])
    got = np.stack([df[c].to_numpy(np.float32) for c in ("y", "x", "mass", "r")], axis=1)
    assert len(got) == len(want) > 0
    # the same set of rows: order both by radius, then position
    g = got[np.lexsort((got[:, 1], got[:, 0], got[:, 3]))]
    w = want[:, :4][np.lexsort((want[:, 1], want[:, 0], want[:, 3]))]
    assert same_floats(g, w)


# characterize_points: oracle table columns / engine columns and the
# reference's ResultRow fields (mass, Rg, raw, signal, ecc)
CP_FIELDS = [("mass", 3, 2), ("Rg", 5, 5), ("raw", 6, 6), ("signal", 7, 7), ("ecc", 8, 8)]


def test_oracle_characterize_points_matches_reference(oracle, golden):
    f = golden["c1_frames"][:1].astype(np.float32)
    pts, want = golden["cp_points"], golden["cp_rows"]
    tab = oracle.characterize_points(trackpy_params(9), f, pts, False, False)
    assert len(tab) == len(want) == len(pts)
    for _, col, field in CP_FIELDS:
        assert same_floats(tab[:, col], want[:, field]), col


@pytest.mark.gpu
def test_engine_characterize_points_matches_reference(golden):
    import pandas as pd
    import gpu_tracking_b200 as gt
    f = golden["c1_frames"][:1]
    pts, want = golden["cp_points"], golden["cp_rows"]
    df = gt.characterize_points(f, pd.DataFrame({"y": pts[:, 0], "x": pts[:, 1]}), diameter=9, tqdm=False)
    assert len(df) == len(want)
    for name, _, field in CP_FIELDS:
        assert same_floats(df[name].to_numpy(), want[:, field]), name
