"""Writes tests/golden/trackpy_ref_64x96.npz and tests/golden/log_ref_48x56.npz:
outputs of the reference's own WGSL shaders (preprocess_rows/cols, max_rows +
extract_max, walk + characterize; separable_log, logspace_max; the frame std
reduction; correct_illumination; adaptive_filter; characterize at given points), translated to C++ by oracle/wgsl2cpp.py and built into
oracle/_ref/ from the reference checkout, on small seeded synthetic frames.

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


if __name__ == "__main__":
    main()
