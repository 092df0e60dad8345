"""Golden vectors of the reference's own post-processing and linking.

tests/golden/postprocess_ref.npz (tests/golden/make_golden.py) holds whole
output tables of the reference's path — its WGSL shaders, then its Rust
post_process (filter_close_trackpy / prune_blobs_log, the doughnut block,
the column layout), its Linker and the duration column — and the ids of its
link_rust / connect_rust paths.  The Rust was translated mechanically from
the reference's source (oracle/rust2py.py) and run on the CPU, so these
fixtures pin the stages that were otherwise checked only by hand-derived
cases.  They need no reference checkout:

* the oracle's C++ restatement reproduces every table, id and duration;
* the engine (-m gpu) reproduces them through its public API.

Comparisons are exact: integer columns equal, float columns bit-identical
(a NaN equals any NaN).  Where the reference checkout was present at build
time (oracle/_ref/rust_ref.py), the translated reference is also compared
with the oracle on randomized inputs, beyond the fixtures.
"""
import os

import numpy as np
import pytest

from gpu_tracking_b200._params import COLUMN_INDEX, log_params, trackpy_params

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "postprocess_ref.npz")
# the generator's cases (tests/golden/make_golden.py: POST_CASES, LINK_CASES, CONNECT_CASES)
POST_CASES = [
    ("trackpy", dict(diameter=9, minmass=300.0, search_range=5.0, memory=1), None),
    ("trackpy", dict(diameter=7, minmass=100.0, separation=6, bg_radius=8.0, gap_radius=1.5, search_range=4.0,
                     memory=2), [1]),
    ("trackpy", dict(diameter=11, minmass=200.0, filter_close=False, doughnut_correction=False, search_range=6.0),
     None),
    ("trackpy", dict(diameter=9, minmass=250.0, characterize=False, search_range=5.0, memory=3), None),
    ("log", dict(min_radius=2.0, max_radius=6.0, n_radii=4, minmass=50.0, search_range=5.0), None),
    ("log", dict(min_radius=2.0, max_radius=6.0, n_radii=5, log_spacing=True, overlap_threshold=0.3, minmass=20.0,
                 search_range=6.0, memory=1), None),
]
LINK_CASES = [(31, 12, 40, 5.0, 0, 0), (32, 15, 50, 5.0, 3, 0), (33, 10, 30, 4.0, 1, 4)]
CONNECT_CASES = [(41, 6, 30, 2.0), (42, 5, 20, 3.0)]
INT_COLUMNS = ("frame", "particle", "duration")


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def case_params(style, kw):
    if style == "trackpy":
        return trackpy_params(**kw)
    kw2 = dict(kw)
    return log_params(kw2.pop("min_radius"), kw2.pop("max_radius"), **kw2)


def case_frames(golden, style):
    return golden["tp_frames"] if style == "trackpy" else golden["log_frames"]


def assert_columns_equal(get, want_table, want_cols, label):
    for j, name in enumerate(want_cols):
        got = get(name)
        want = want_table[:, j]
        if name in INT_COLUMNS:
            g, w = np.asarray(got).astype(np.int64), want.astype(np.int64)
            bad = np.flatnonzero(g != w)
        else:
            g, w = np.asarray(got, np.float32), want.astype(np.float32)
            same = (g.view(np.uint32) == w.view(np.uint32)) | (np.isnan(g) & np.isnan(w))
            bad = np.flatnonzero(~same)
        assert bad.size == 0, "%s: column %s differs at %d rows (first %s): got %r want %r" % (
            label, name, bad.size, bad[:5], g[bad[:5]], w[bad[:5]])


# ------------------------------------------------------------------ oracle
@pytest.mark.parametrize("case", range(len(POST_CASES)))
def test_oracle_tables_match_reference_post_processing(oracle, golden, case):
    style, kw, reset = POST_CASES[case]
    p = case_params(style, kw)
    frames = case_frames(golden, style).astype(np.float32)
    tab = oracle.batch(p, frames, reset_points=reset)
    want = golden["post%d_table" % case]
    cols = [str(c) for c in golden["post%d_columns" % case]]
    assert len(tab) == len(want) and len(want) > 0
    assert_columns_equal(lambda n: tab[:, COLUMN_INDEX[n]], want, cols, "oracle case %d" % case)


@pytest.mark.parametrize("case", range(len(LINK_CASES)))
def test_oracle_link_matches_reference_linker(oracle, golden, case):
    R, mem = LINK_CASES[case][3], LINK_CASES[case][4]
    ids = oracle.link(golden["link%d_rows" % case], R, mem)
    assert np.array_equal(ids, golden["link%d_ids" % case])


@pytest.mark.parametrize("case", range(len(CONNECT_CASES)))
def test_oracle_connect_matches_reference(oracle, golden, case):
    R = CONNECT_CASES[case][3]
    ia, ib = oracle.connect(golden["connect%d_a" % case], golden["connect%d_b" % case], R)
    assert np.array_equal(ia, golden["connect%d_ia" % case])
    assert np.array_equal(ib, golden["connect%d_ib" % case])


# ------------------------------------------------------------------ engine
@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(POST_CASES)))
def test_engine_tables_match_reference_post_processing(golden, case):
    import gpu_tracking_b200 as gt
    style, kw, reset = POST_CASES[case]
    frames = case_frames(golden, style)
    kw = dict(kw)
    if reset is not None:
        kw["linker_reset_points"] = reset
    if style == "trackpy":
        d = kw.pop("diameter")
        df = gt.batch(frames, d, tqdm=False, **kw)
    else:
        lo, hi = kw.pop("min_radius"), kw.pop("max_radius")
        df = gt.LoG(frames, lo, hi, tqdm=False, **kw)
    want = golden["post%d_table" % case]
    cols = [str(c) for c in golden["post%d_columns" % case]]
    assert list(df.columns) == cols
    assert len(df) == len(want) and len(want) > 0
    assert_columns_equal(lambda n: df[n].to_numpy(), want, cols, "engine case %d" % case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(LINK_CASES)))
def test_engine_link_matches_reference_linker(golden, case):
    import gpu_tracking_b200 as gt
    R, mem = LINK_CASES[case][3], LINK_CASES[case][4]
    ids = gt.link(golden["link%d_rows" % case], R, mem)
    assert np.array_equal(np.asarray(ids, np.int64), golden["link%d_ids" % case])


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CONNECT_CASES)))
def test_engine_connect_matches_reference(golden, case):
    import pandas as pd

    import gpu_tracking_b200 as gt
    R = CONNECT_CASES[case][3]
    a, b = golden["connect%d_a" % case], golden["connect%d_b" % case]
    da = pd.DataFrame(a, columns=["frame", "y", "x"])
    db = pd.DataFrame(b, columns=["frame", "y", "x"])
    ia, ib = gt.connect(da, db, R, merge=False)
    assert np.array_equal(ia["connect particle"].to_numpy(np.int64), golden["connect%d_ia" % case])
    assert np.array_equal(ib["connect particle"].to_numpy(np.int64), golden["connect%d_ib" % case])


# ------------------------------------------------- translated reference (CPU)
def _ref_post():
    from oracle import ref_post
    if not ref_post.available():
        pytest.skip("the reference checkout was absent when the oracle was built")
    return ref_post


def _detections(seed, T, n, R, size, first_frame=0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, size, (n, 2))
    rows = []
    for t in range(T):
        keep = rng.random(n) > 0.05
        for k in np.flatnonzero(keep):
            rows.append((first_frame + t, pos[k, 0], pos[k, 1]))
        pos = pos + rng.normal(0, R / 3, pos.shape)
        dead = rng.random(n) < 0.1
        pos[dead] = rng.uniform(0, size, (dead.sum(), 2))
    return np.array(rows, np.float32)


def test_fixture_is_what_the_reference_produces(golden):
    """The committed fixture equals a fresh run of the translated reference."""
    rp = _ref_post()
    style, kw, reset = POST_CASES[0]
    table, cols = rp.batch(case_params(style, kw), case_frames(golden, style).astype(np.float32), reset)
    assert np.array_equal(table.view(np.uint32), golden["post0_table"].view(np.uint32))
    R, mem = LINK_CASES[1][3], LINK_CASES[1][4]
    assert np.array_equal(rp.link(golden["link1_rows"], R, mem), golden["link1_ids"])


@pytest.mark.parametrize("seed", range(6))
def test_oracle_linker_equals_reference_linker_randomized(oracle, seed):
    rp = _ref_post()
    rng = np.random.default_rng(seed)
    R = float(rng.uniform(3.0, 6.0))
    mem = int(rng.integers(0, 4))
    rows = _detections(500 + seed, int(rng.integers(6, 14)), int(rng.integers(20, 50)), R, 110.0,
                       first_frame=int(rng.integers(0, 3)))
    if seed % 3 == 2:
        rows[rng.integers(0, len(rows), 3), 0] = np.nan   # NaN frames join the group in progress
    assert np.array_equal(oracle.link(rows, R, mem), rp.link(rows, R, mem))


def test_oracle_and_reference_raise_the_same_errors(oracle):
    rp = _ref_post()
    import rust_rt
    rng = np.random.default_rng(0)
    n = 72   # one subnet with load 72 * 72 = 5184 > 5000
    rows = np.r_[np.c_[np.zeros(n), rng.uniform(0, 1, (n, 2))], np.c_[np.ones(n), rng.uniform(0, 1, (n, 2))]]
    with pytest.raises(rust_rt.RustError) as e:
        rp.link(rows, 5.0, 0)
    assert e.value.kind == "TooDenseToLink"
    with pytest.raises(oracle.OracleError) as e2:
        oracle.link(rows, 5.0, 0)
    assert e2.value.code == 8
    unsorted = np.array([[1, 0, 0], [0, 1, 1]], np.float32)
    with pytest.raises(rust_rt.RustError) as e:
        rp.link(unsorted, 2.0, 0)
    assert e.value.kind == "NonSortedCharacterization"
    with pytest.raises(oracle.OracleError) as e2:
        oracle.link(unsorted, 2.0, 0)
    assert e2.value.code == 4


@pytest.mark.parametrize("seed", range(3))
def test_oracle_connect_equals_reference_randomized(oracle, seed):
    rp = _ref_post()
    rng = np.random.default_rng(seed)
    a = _detections(700 + seed, 5, 25, 2.0, 50.0)
    b = a[rng.random(len(a)) > 0.3].copy()
    b[:, 1:] += rng.normal(0, 1.0, (len(b), 2)).astype(np.float32)
    if seed == 1:
        b = b[b[:, 0] != 2]   # a frame only one side has
    ia, ib = oracle.connect(a, b, 2.0)
    ra, rb = rp.connect(a, b, 2.0)
    assert np.array_equal(ia, ra) and np.array_equal(ib, rb)


@pytest.mark.parametrize("seed", range(4))
def test_oracle_batch_equals_reference_randomized(oracle, seed):
    rp = _ref_post()
    from synth import video
    rng = np.random.default_rng(seed)
    if seed < 3:
        frames, _ = video(4, 56, 72, 18, seed=800 + seed, D=1.0)
        kw = dict(diameter=int(rng.choice([7, 9, 11])), minmass=float(rng.uniform(100, 300)),
                  search_range=float(rng.uniform(3, 6)), memory=int(rng.integers(0, 3)),
                  filter_close=bool(seed != 1), separation=int(rng.integers(5, 12)))
        p = trackpy_params(**kw)
        frames = frames.astype(np.float32)
    else:
        frames, _ = video(3, 40, 48, 8, seed=900, dtype=np.float32, read_noise=5.0, bg=50.0, sigma_range=(1.4, 4.0))
        p = log_params(2.0, 6.0, n_radii=4, log_spacing=True, overlap_threshold=0.5, minmass=30.0, search_range=5.0)
    want, cols = rp.batch(p, frames)
    tab = oracle.batch(p, frames)
    assert len(tab) == len(want)
    assert_columns_equal(lambda n: tab[:, COLUMN_INDEX[n]], want, cols, "randomized %d" % seed)
