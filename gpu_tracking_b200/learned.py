"""Learned walk seeds: a small BF16 network proposes where the centroid walk
starts, in place of the bandpass local maxima.

Not part of the reference's API.  The network (4 layers of 3x3 convolutions,
32 channels, over 4x4-pixel cells; about 24k parameters) is trained on the
GPU by the engine's own forward and backward kernels, on crops labelled by
the plain method's converged detections.  In ``batch_learned`` each proposal
seeds the plain walk, which runs to its own convergence criterion from there;
characterization, filter_close, the doughnut correction and linking are the
plain method's, so a detection whose walk ends where the plain one does is
identical to it in every column.  ``compare`` scores a learned table against
the plain one (recall, precision, added position error).
"""
import ctypes

import numpy as np

from . import _ffi
from ._params import trackpy_params
from .api import _DEVICE, _Frames, _run, _table_to_frame

__all__ = ["ProposalNet", "batch_learned", "compare", "calibrate"]

_P32 = ctypes.POINTER(ctypes.c_float)
_P64 = ctypes.POINTER(ctypes.c_int64)


class ProposalNet:
    """The proposal network on the engine's device."""

    def __init__(self, seed=0):
        self._ctx = _ffi.context(_DEVICE)
        self._h = ctypes.c_void_p()
        self._ctx.check(_ffi.lib().gt_proposal_create(self._ctx.handle, int(seed), ctypes.byref(self._h)))

    @staticmethod
    def num_params():
        return int(_ffi.lib().gt_proposal_num_params())

    @property
    def handle(self):
        return self._h

    def _get(self):
        p = np.empty(self.num_params(), np.float32)
        m, s, t = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        self._ctx.check(_ffi.lib().gt_proposal_get(self._ctx.handle, self._h, p.ctypes.data_as(_P32), ctypes.byref(m),
                                                   ctypes.byref(s), ctypes.byref(t)))
        return p, m.value, s.value, t.value

    def _set(self, params=None, mean=None, scale=None, threshold=None):
        _, m, s, t = self._get()
        m = m if mean is None else mean
        s = s if scale is None else scale
        t = t if threshold is None else threshold
        ptr = None
        if params is not None:
            params = np.ascontiguousarray(params, np.float32)
            if params.shape != (self.num_params(),):
                raise ValueError("expected %d parameters" % self.num_params())
            ptr = params.ctypes.data_as(_P32)
        self._ctx.check(_ffi.lib().gt_proposal_set(self._ctx.handle, self._h, ptr, float(m), float(s), float(t)))

    @property
    def params(self):
        return self._get()[0]

    @params.setter
    def params(self, value):
        self._set(params=value)

    @property
    def mean(self):
        return self._get()[1]

    @property
    def scale(self):
        return self._get()[2]

    @property
    def threshold(self):
        """Score logit a cell must exceed to propose a seed."""
        return self._get()[3]

    @threshold.setter
    def threshold(self, value):
        self._set(threshold=float(value))

    def set_normalization(self, mean, scale):
        self._set(mean=float(mean), scale=float(scale))

    def fit_normalization(self, frames, max_frames=8):
        """Input normalisation from the first frames: (pixel - mean) / std."""
        if hasattr(frames, "is_cuda"):
            sample = frames[:max_frames].float()
            mean, std = float(sample.mean()), float(sample.std())
        else:
            sample = np.asarray(frames[:max_frames], np.float64)
            mean, std = float(sample.mean()), float(sample.std())
        self.set_normalization(mean, 1.0 / max(std, 1e-6))

    def train(self, frames, labels, steps=800, batch=256, crop=128, lr=3e-3, pos_weight=8.0, offset_weight=1.0,
              seed=1):
        """Train on random crops of ``frames`` labelled by ``labels`` (a table
        with frame, y, x columns, frame = index into ``frames``).  Returns the
        per-step (score loss, offset loss), shape (steps, 2)."""
        fr = _Frames(frames)
        if self.scale == 1.0 and self.mean == 0.0:
            self.fit_normalization(frames)
        lf = np.ascontiguousarray(np.asarray(labels["frame"]), np.int64)
        ly = np.ascontiguousarray(np.asarray(labels["y"]), np.float32)
        lx = np.ascontiguousarray(np.asarray(labels["x"]), np.float32)
        o = _ffi.TrainOpts()
        _ffi.lib().gt_train_opts_default(ctypes.byref(o))
        o.steps, o.batch, o.crop = int(steps), int(batch), int(crop)
        o.lr, o.pos_weight, o.offset_weight, o.seed = float(lr), float(pos_weight), float(offset_weight), int(seed)
        loss = np.zeros((max(int(steps), 0), 2), np.float32)
        self._ctx.check(_ffi.lib().gt_proposal_train(
            self._ctx.handle, self._h, fr.ptr, fr.dtype, fr.T, fr.H, fr.W, lf.ctypes.data_as(_P64),
            ly.ctypes.data_as(_P32), lx.ctypes.data_as(_P32), len(lf), ctypes.byref(o),
            loss.ctypes.data_as(_P32) if len(loss) else None))
        return loss

    def maps(self, frames):
        """Per-cell outputs (T, ceil(H/4), ceil(W/4), 4): score logit, row and
        column offset of the detection from the cell centre, 0."""
        fr = _Frames(frames)
        out = np.zeros((fr.T, (fr.H + 3) // 4, (fr.W + 3) // 4, 4), np.float32)
        self._ctx.check(_ffi.lib().gt_proposal_maps(self._ctx.handle, self._h, fr.ptr, fr.dtype, fr.T, fr.H, fr.W,
                                                    out.ctypes.data_as(_P32)))
        return out

    def save(self, path):
        p, m, s, t = self._get()
        np.savez(path, params=p, mean=m, scale=s, threshold=t)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        net = cls()
        net._set(params=z["params"], mean=float(z["mean"]), scale=float(z["scale"]), threshold=float(z["threshold"]))
        return net

    def close(self):
        if self._h:
            _ffi.lib().gt_proposal_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_learned(file_or_array, diameter, net, **kwargs):
    """``batch`` with the network's seeds instead of the bandpass local maxima.

    Same arguments and output columns as ``batch`` (trackpy style); snr,
    minmass_snr, adaptive_background and illumination correction are not
    supported with learned seeds."""
    params = trackpy_params(diameter, **kwargs)
    ctx = _ffi.context(_DEVICE)
    fr = _Frames(file_or_array, kwargs.get("frames"))
    fn = fr.frame_numbers
    reset = kwargs.get("linker_reset_points")
    reset_arr = np.asarray(list(reset) if reset is not None else [], np.int64)
    out = ctypes.c_void_p()

    def call():
        return _ffi.lib().gt_batch_learned(ctx.handle, ctypes.byref(params), net.handle, fr.ptr, fr.dtype, fr.T, fr.H,
                                           fr.W, fn.ctypes.data_as(_P64) if fn is not None else None,
                                           reset_arr.ctypes.data_as(_P64) if len(reset_arr) else None,
                                           len(reset_arr), ctypes.byref(out))

    st = _run(ctx, call, bool(kwargs.get("tqdm", True)) and fr.T > 1)
    ctx.check(st)
    return _table_to_frame(ctx, out, params)


def last_walk_starts():
    """Walk starts (candidates or seeds) of the last batch / batch_learned call."""
    return int(_ffi.lib().gt_last_walk_starts(_ffi.context(_DEVICE).handle))


def compare(plain, learned, tol=0.5):
    """Score learned detections against the plain method's, frame by frame.

    A plain detection is found when a learned one lies within ``tol`` pixels
    (nearest first, one-to-one).  Returns recall, precision, the matched
    count, how many matched rows sit at the same position (bit for bit) and
    how many are identical in every column the two tables share, and the mean
    and maximum added position error (pixels)."""
    from scipy.spatial import cKDTree
    cols = [c for c in plain.columns if c in learned.columns and c not in ("particle", "duration")]
    iy, ix = cols.index("y"), cols.index("x")
    vp_all = plain[cols].to_numpy(np.float32)
    vl_all = learned[cols].to_numpy(np.float32)
    fp = plain["frame"].to_numpy()
    fl = learned["frame"].to_numpy()
    op, ol = np.argsort(fp, kind="stable"), np.argsort(fl, kind="stable")
    up, sp = np.unique(fp[op], return_index=True)
    ul, sl = np.unique(fl[ol], return_index=True)
    ep, el = np.append(sp[1:], len(op)), np.append(sl[1:], len(ol))
    lpos = {f: (a, b) for f, a, b in zip(ul, sl, el)}
    pi_all, li_all, d_all = [], [], []
    for f, a, b in zip(up, sp, ep):
        if f not in lpos:
            continue
        la, lb = lpos[f]
        ip, il = op[a:b], ol[la:lb]
        tree = cKDTree(vl_all[il][:, [iy, ix]].astype(np.float64))
        d, j = tree.query(vp_all[ip][:, [iy, ix]].astype(np.float64), distance_upper_bound=tol)
        ok = np.isfinite(d)
        ip, d, j = ip[ok], d[ok], j[ok]
        order = np.argsort(d, kind="stable")
        _, first = np.unique(j[order], return_index=True)
        keep = order[first]
        pi_all.append(ip[keep])
        li_all.append(il[j[keep]])
        d_all.append(d[keep])
    if pi_all:
        pi, li, d = np.concatenate(pi_all), np.concatenate(li_all), np.concatenate(d_all)
    else:
        pi = li = np.zeros(0, np.int64)
        d = np.zeros(0)
    a, b = vp_all[pi], vl_all[li]
    same_pos = (a[:, iy] == b[:, iy]) & (a[:, ix] == b[:, ix])
    same_all = np.all((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b)), axis=1)
    n_plain, n_learned, matched = len(plain), len(learned), len(pi)
    return {
        "recall": matched / n_plain if n_plain else 1.0,
        "precision": matched / n_learned if n_learned else 1.0,
        "matched": int(matched),
        "identical": int(same_all.sum()),
        "same_position": int(same_pos.sum()),
        "plain": n_plain,
        "learned": n_learned,
        "mean_position_error": float(d.mean()) if matched else 0.0,
        "max_position_error": float(d.max()) if matched else 0.0,
    }


def calibrate(net, frames, diameter, plain=None, recall=0.997, thresholds=None, **kwargs):
    """Highest score threshold whose learned table reaches ``recall`` of the
    plain method's detections on ``frames`` (else the one with the best
    recall); sets it on ``net`` and returns (threshold, [(threshold, recall,
    precision)] for every threshold tried)."""
    from .api import batch
    kw = {k: v for k, v in kwargs.items() if k not in ("search_range", "memory")}
    kw["tqdm"] = False
    if plain is None:
        plain = batch(frames, diameter, **kw)
    if len(plain) == 0:
        raise ValueError("the plain method finds nothing in the calibration frames")
    if thresholds is None:
        thresholds = np.arange(2.0, -6.01, -0.5)
    curve = []
    chosen = None
    for t in thresholds:
        net.threshold = float(t)
        s = compare(plain, batch_learned(frames, diameter, net, **kw))
        curve.append((float(t), s["recall"], s["precision"]))
        if s["recall"] >= recall:
            chosen = float(t)
            break
    if chosen is None:
        best = max(r for _, r, _ in curve)
        chosen = next(t for t, r, _ in curve if r == best)
    net.threshold = chosen
    return chosen, curve
