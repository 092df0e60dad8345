"""Writes tests/golden/trackpy_ref_64x96.npz: outputs of the reference's own
WGSL shaders (preprocess_rows/cols, max_rows + extract_max, walk +
characterize), translated to C++ by oracle/wgsl2cpp.py and built into
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

from gpu_tracking_b200._params import trackpy_params  # noqa: E402
from oracle import loader  # noqa: E402
from synth import video  # noqa: E402

# (keyword arguments of batch, generator seed)
CASES = [
    (dict(diameter=9, minmass=300.0, separation=9), 11),
    (dict(diameter=11, minmass=200.0), 12),
    (dict(diameter=7, minmass=0.0, truncate_preprocessed=False), 13),
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
            proc = loader.ref_preprocess(p, f)
            cands = loader.ref_candidates(p, proc)
            rows = loader.ref_walk(p, proc, f, cands, characterize=True)
            if t == 0:
                out["c%d_t%d_processed" % (c, t)] = proc
            out["c%d_t%d_candidates" % (c, t)] = cands
            out["c%d_t%d_rows" % (c, t)] = rows
    path = os.path.join(HERE, "trackpy_ref_64x96.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
