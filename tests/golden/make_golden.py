"""Writes tests/golden/trackpy_ref_64x96.npz and tests/golden/log_ref_48x56.npz:
outputs of the reference's own WGSL shaders (preprocess_rows/cols, max_rows +
extract_max, walk + characterize; separable_log, logspace_max; the frame std
reduction; correct_illumination; adaptive_filter; characterize at given points), translated to C++ by oracle/wgsl2cpp.py and built into
oracle/_ref/ from the reference checkout, on small seeded synthetic frames.

It also writes tests/golden/postprocess_ref.npz: whole tables (every column,
particle ids and durations) of the reference's own path — its shaders, then
its Rust post-processing (filter_close_trackpy, prune_blobs_log, the
doughnut block, column layout) and its Linker — with the Rust translated to
Python by oracle/rust2py.py (oracle/_ref/rust_ref.py) and driven by
oracle/ref_post.py; and the particle ids of its link_rust / connect_rust
paths (linker_all, connect_all) on seeded detection sets.

The fixtures let the oracle and the GPU path be checked against the
reference's shaders on machines that have no reference checkout.  Run from
the repository root after building the oracle and its reference translation:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from gpu_tracking_b200._params import log_params, trackpy_params  # noqa: E402
from oracle import loader  # noqa: E402
from synth import video  # noqa: E402

# (keyword arguments of batch, generator seed)
CASES = [
    (dict(diameter=9, minmass=300.0, separation=9), 11),
    (dict(diameter=11, minmass=200.0), 12),
    (dict(diameter=7, minmass=0.0, truncate_preprocessed=False), 13),
    # thresholds from the frame std: extract_max.wgsl:37 and walk.wgsl:200-205
    (dict(diameter=9, snr=1.2, minmass_snr=0.3), 14),
    # per-frame illumination correction: every stage sees frame / smoothed frame
    (dict(diameter=9, minmass=0.05, illumination_sigma=4.0, illumination_correction_per_frame=True), 15),
    # adaptive_background: two adaptive_filter passes over the walked rows
    (dict(diameter=9, adaptive_background=2, snr=0.3, minmass_snr=1.0), 16),
]
T, H, W = 2, 64, 96


def main():
    if not loader.ref_available():
        raise SystemExit("the reference translation (oracle/_ref) is not built")
    out = {}
    for c, (kw, seed) in enumerate(CASES):
        frames, _ = video(T, H, W, 14, seed=seed)
        out["c%d_frames" % c] = frames.astype(np.uint16)
        p = trackpy_params(**kw)
        for t in range(T):
            f = frames[t].astype(np.float32)
            if kw.get("illumination_correction_per_frame"):
                f = loader.ref_illumination(p, f, np.float32(kw["illumination_sigma"]), f)[1]
            proc = loader.ref_preprocess(p, f)
            std = loader.ref_frame_std(f) if ("snr" in kw or "minmass_snr" in kw) else 0.0
            cands = loader.ref_candidates(p, proc, pic_std=std)
            rows = loader.ref_walk(p, proc, f, cands, characterize=True, pic_std=std)
            if kw.get("adaptive_background"):
                rows = loader.ref_adaptive(p, f, rows, kw["adaptive_background"], std)
            if t == 0:
                out["c%d_t%d_processed" % (c, t)] = proc
            out["c%d_t%d_candidates" % (c, t)] = cands
            out["c%d_t%d_rows" % (c, t)] = rows
        # the reference's frame std (snr / minmass_snr thresholds)
        out["c%d_std" % c] = np.array([loader.ref_frame_std(frames[t].astype(np.float32)) for t in range(T)],
                                      np.float32)
    # characterize_points: the reference's characterize shader at given points
    f = out["c1_frames"][0].astype(np.float32)
    p = trackpy_params(9)
    rng = np.random.default_rng(3)
    pts = np.c_[rng.uniform(0, 63, 25), rng.uniform(0, 95, 25)].astype(np.float32)
    pts[:3] = [[10.5, 20.5], [11.5, 21.5], [0.0, 0.0]]   # half-way rounding and a corner
    out["cp_points"] = pts
    out["cp_rows"] = loader.ref_characterize_points(p, loader.ref_preprocess(p, f), f, pts)
    path = os.path.join(HERE, "trackpy_ref_64x96.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")

    # LoG: the scale planes of every radius, the scale-space maxima and their walks
    out = {}
    frames, _ = video(1, 48, 56, 10, seed=7, dtype=np.float32, read_noise=5.0, bg=50.0)
    f = frames[0]
    out["frame"] = f
    for s_, spacing in enumerate((False, True)):
        p = log_params(2.0, 6.0, n_radii=4, log_spacing=spacing)
        planes, radii = loader.log_planes(p, f)   # radii only: the planes below are the reference's
        proc = loader.ref_preprocess(p, f)
        ref_planes = np.stack([loader.ref_laplace(p, f, np.float32(r) / np.sqrt(np.float32(2.0))) for r in radii])
        out["s%d_radii" % s_] = radii
        out["s%d_planes" % s_] = ref_planes
        n = len(radii)
        for i in range(n):
            edge = -1 if i == 0 else (1 if i == n - 1 else 0)
            bottom = ref_planes[i - 1] if i > 0 else np.zeros_like(f)
            top = ref_planes[i + 1] if i < n - 1 else np.zeros_like(f)
            cands = loader.ref_logspace_max(p, bottom, ref_planes[i], top, proc, edge, radii[i])
            out["s%d_r%d_candidates" % (s_, i)] = cands
            out["s%d_r%d_rows" % (s_, i)] = loader.ref_walk(p, proc, f, cands, r=float(radii[i]), characterize=False)
    path = os.path.join(HERE, "log_ref_48x56.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


# whole-path cases: (style, keyword arguments, linker_reset_points)
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
# link_rust / connect_rust cases: (seed, frames, points, search_range, memory, first frame)
LINK_CASES = [(31, 12, 40, 5.0, 0, 0), (32, 15, 50, 5.0, 3, 0), (33, 10, 30, 4.0, 1, 4)]
CONNECT_CASES = [(41, 6, 30, 2.0), (42, 5, 20, 3.0)]


def detections(seed, T, n, R, size, first_frame=0):
    """Seeded (frame, y, x) rows: n points doing Brownian steps of R/3,
    5 % missing per frame, 10 % replaced by new points per frame."""
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


def post_main():
    from oracle import ref_post
    if not ref_post.available():
        raise SystemExit("the reference's Rust translation (oracle/_ref/rust_ref.py) is not built")
    out = {}
    tp_frames, _ = video(6, 64, 80, 22, seed=21, D=0.8)
    log_frames, _ = video(4, 48, 56, 10, seed=22, dtype=np.float32, read_noise=5.0, bg=50.0,
                          sigma_range=(1.4, 4.0), D=0.5)
    out["tp_frames"] = tp_frames.astype(np.uint16)
    out["log_frames"] = log_frames
    for c, (style, kw, reset) in enumerate(POST_CASES):
        if style == "trackpy":
            p = trackpy_params(**kw)
            frames = tp_frames.astype(np.float32)
        else:
            kw2 = dict(kw)
            p = log_params(kw2.pop("min_radius"), kw2.pop("max_radius"), **kw2)
            frames = log_frames
        table, cols = ref_post.batch(p, frames, linker_reset_points=reset)
        out["post%d_table" % c] = table
        out["post%d_columns" % c] = np.array(cols)
    for c, (seed, T, n, R, mem, first) in enumerate(LINK_CASES):
        rows = detections(seed, T, n, R, 100.0, first)
        out["link%d_rows" % c] = rows
        out["link%d_ids" % c] = ref_post.link(rows, R, mem)
    for c, (seed, T, n, R) in enumerate(CONNECT_CASES):
        a = detections(seed, T, n, R, 60.0)
        b = a.copy()
        rng = np.random.default_rng(seed)
        b[:, 1:] += rng.normal(0, R / 2, (len(b), 2)).astype(np.float32)
        b = b[rng.random(len(b)) > 0.2]
        out["connect%d_a" % c] = a
        out["connect%d_b" % c] = b
        ia, ib = ref_post.connect(a, b, R)
        out["connect%d_ia" % c] = ia
        out["connect%d_ib" % c] = ib
    path = os.path.join(HERE, "postprocess_ref.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
    post_main()
