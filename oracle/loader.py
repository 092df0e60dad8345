"""ctypes front end of the oracle (test infrastructure only).

``lib()`` is the C++ restatement (oracle/gt_oracle.cpp); ``ref()`` is the
reference's own WGSL shaders translated to C++ (oracle/_ref/, built from the
reference checkout by ``make ref``).  Everything here is a checker: only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

c_f32p = ctypes.POINTER(ctypes.c_float)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_f64p = ctypes.POINTER(ctypes.c_double)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def reference_root():
    """The reference checkout: $GT_REFERENCE_ROOT, else a ``reference``
    directory beside this repository's root."""
    env = os.environ.get("GT_REFERENCE_ROOT")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def build():
    """Compile the oracle (and the reference translation when the checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = reference_root()
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + ref], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "libgt_oracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.oracle_gpu_params.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp]
        L.oracle_params_sizeof.restype = ctypes.c_int32
        L.oracle_log_radii.argtypes = [vp, c_f32p]
        L.oracle_preprocess.argtypes = [vp, c_f32p, ctypes.c_int32, ctypes.c_int32, c_f32p]
        L.oracle_candidates.argtypes = [vp, c_f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, c_i32p,
                                        ctypes.c_int64]
        L.oracle_candidates.restype = ctypes.c_int64
        L.oracle_walk.argtypes = [vp, c_f32p, c_f32p, ctypes.c_int32, ctypes.c_int32, c_i32p, ctypes.c_int64,
                                  ctypes.c_float, ctypes.c_float, c_f32p, c_i32p]
        L.oracle_frame_std.argtypes = [c_f32p, ctypes.c_int64, ctypes.c_uint32, c_f32p]
        L.oracle_adaptive.argtypes = [vp, c_f32p, ctypes.c_int32, ctypes.c_int32, c_f32p, ctypes.c_int64,
                                      ctypes.c_uint32, ctypes.c_float, ctypes.c_int32, c_f32p]
        L.oracle_adaptive.restype = ctypes.c_int64
        L.oracle_smooth_profile.argtypes = [c_f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, c_f32p]
        L.oracle_log_planes.argtypes = [vp, c_f32p, ctypes.c_int32, ctypes.c_int32, c_f32p, c_f32p]
        L.oracle_batch.argtypes = [vp, c_f32p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, c_i64p, c_i64p,
                                   ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(vp)]
        L.oracle_characterize_points.argtypes = [vp, c_f32p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                 c_f32p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.POINTER(vp)]
        L.oracle_table_nrows.argtypes = [vp]
        L.oracle_table_nrows.restype = ctypes.c_int64
        L.oracle_table_get.argtypes = [vp, c_f64p]
        L.oracle_table_free.argtypes = [vp]
        L.oracle_link.argtypes = [c_f32p, ctypes.c_int64, ctypes.c_float, ctypes.c_uint32, c_i64p]
        L.oracle_connect.argtypes = [c_f32p, ctypes.c_int64, c_f32p, ctypes.c_int64, ctypes.c_float, c_i64p,
                                     c_i64p]
        _LIB = L
    return _LIB


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libgt_ref.so"))


def ref():
    global _REF
    if _REF is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libgt_ref.so"))
        vp = ctypes.c_void_p
        L.ref_preprocess.argtypes = [vp, ctypes.c_int32, c_f32p, c_f32p]
        L.ref_candidates.argtypes = [vp, c_f32p, ctypes.c_float, c_i32p, ctypes.c_int64]
        L.ref_candidates.restype = ctypes.c_int64
        L.ref_walk.argtypes = [vp, c_f32p, c_f32p, c_i32p, ctypes.c_int64, ctypes.c_float, ctypes.c_float,
                               ctypes.c_int32, c_f32p]
        L.ref_walk.restype = ctypes.c_int64
        L.ref_characterize_points.argtypes = [vp, c_f32p, c_f32p, c_f32p, ctypes.c_int64]
        L.ref_laplace.argtypes = [vp, c_f32p, ctypes.c_float, c_f32p]
        L.ref_logspace_max.argtypes = [vp, c_f32p, c_f32p, c_f32p, c_f32p, ctypes.c_float, ctypes.c_int32,
                                       ctypes.c_float, c_i32p, ctypes.c_int64]
        L.ref_logspace_max.restype = ctypes.c_int64
        L.ref_frame_std.argtypes = [c_f32p, ctypes.c_int64, ctypes.c_uint32, c_f32p]
        L.ref_frame_std.restype = ctypes.c_float
        L.ref_adaptive.argtypes = [vp, c_f32p, c_f32p, ctypes.c_int64, ctypes.c_uint32, ctypes.c_float, ctypes.c_int32,
                                   c_f32p, c_f32p]
        L.ref_adaptive.restype = ctypes.c_int64
        L.ref_illumination.argtypes = [vp, c_f32p, ctypes.c_float, c_f32p, c_f32p]
        _REF = L
    return _REF


class OracleError(RuntimeError):
    def __init__(self, code):
        super().__init__("oracle status %d" % code)
        self.code = code


def _check(st):
    if st != 0:
        raise OracleError(st)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------------ oracle
def gpu_params(p, H, W):
    buf = (ctypes.c_int32 * 16)()
    lib().oracle_gpu_params(ctypes.byref(p), H, W, buf)
    return buf


def log_radii(p):
    out = np.zeros(max(1, p.n_radii), np.float32)
    n = lib().oracle_log_radii(ctypes.byref(p), _ptr(out, c_f32p))
    return out[:n]


def preprocess(p, frame):
    frame = _f32(frame)
    H, W = frame.shape
    out = np.empty_like(frame)
    _check(lib().oracle_preprocess(ctypes.byref(p), _ptr(frame, c_f32p), H, W, _ptr(out, c_f32p)))
    return out


def candidates(p, processed, pic_std=0.0):
    processed = _f32(processed)
    H, W = processed.shape
    cap = H * W
    uv = np.empty((cap, 2), np.int32)
    n = lib().oracle_candidates(ctypes.byref(p), _ptr(processed, c_f32p), H, W, pic_std, _ptr(uv, c_i32p), cap)
    return uv[:n].copy()


def walk(p, processed, raw, uv, r=-1.0, pic_std=0.0):
    processed, raw = _f32(processed), _f32(raw)
    H, W = processed.shape
    uv = np.ascontiguousarray(uv, np.int32)
    n = len(uv)
    rows = np.zeros((max(n, 1), 10), np.float32)
    keep = np.zeros(max(n, 1), np.int32)
    _check(lib().oracle_walk(ctypes.byref(p), _ptr(processed, c_f32p), _ptr(raw, c_f32p), H, W,
                             _ptr(uv, c_i32p), n, r, pic_std, _ptr(rows, c_f32p), _ptr(keep, c_i32p)))
    return rows[:n], keep[:n].astype(bool)


def frame_std(frame, divisor=None):
    """The reference's frame std (StdArray); masked pixels hold the 0xFFFFFFFF pattern."""
    frame = _f32(frame).ravel()
    out = ctypes.c_float()
    _check(lib().oracle_frame_std(_ptr(frame, c_f32p), frame.size, frame.size if divisor is None else divisor,
                                  ctypes.byref(out)))
    return np.float32(out.value)


def smooth_profile(frame, sigma):
    frame = _f32(frame)
    H, W = frame.shape
    out = np.empty_like(frame)
    _check(lib().oracle_smooth_profile(_ptr(frame, c_f32p), H, W, sigma, _ptr(out, c_f32p)))
    return out


def adaptive(p, frame, rows, n_iter, std0, recompute=True):
    frame = _f32(frame)
    H, W = frame.shape
    rows = _f32(rows).reshape(-1, 10)
    out = np.zeros((max(len(rows), 1), 10), np.float32)
    n = lib().oracle_adaptive(ctypes.byref(p), _ptr(frame, c_f32p), H, W, _ptr(rows, c_f32p), len(rows), n_iter,
                              std0, int(recompute), _ptr(out, c_f32p))
    return out[:n].copy()


def log_planes(p, frame):
    frame = _f32(frame)
    H, W = frame.shape
    planes = np.empty((p.n_radii, H, W), np.float32)
    radii = np.empty(p.n_radii, np.float32)
    _check(lib().oracle_log_planes(ctypes.byref(p), _ptr(frame, c_f32p), H, W, _ptr(planes, c_f32p),
                                   _ptr(radii, c_f32p)))
    return planes, radii


def _table(handle):
    L = lib()
    n = L.oracle_table_nrows(handle)
    out = np.empty((n, 16), np.float64)
    if n:
        L.oracle_table_get(handle, _ptr(out, c_f64p))
    L.oracle_table_free(handle)
    return out


def batch(p, frames, frame_numbers=None, reset_points=None, nthreads=0):
    """Full pipeline; returns an (n, 16) float64 table in gt_column order."""
    frames = _f32(frames)
    T, H, W = frames.shape
    fn = None if frame_numbers is None else np.ascontiguousarray(frame_numbers, np.int64)
    rp = np.ascontiguousarray(reset_points if reset_points is not None else [], np.int64)
    h = ctypes.c_void_p()
    _check(lib().oracle_batch(ctypes.byref(p), _ptr(frames, c_f32p), T, H, W,
                              None if fn is None else _ptr(fn, c_i64p), _ptr(rp, c_i64p) if len(rp) else None,
                              len(rp), nthreads, ctypes.byref(h)))
    return _table(h)


def characterize_points(p, frames, points, has_frames, has_r, nthreads=0):
    frames = _f32(frames)
    T, H, W = frames.shape
    pts = _f32(points)
    h = ctypes.c_void_p()
    _check(lib().oracle_characterize_points(ctypes.byref(p), _ptr(frames, c_f32p), T, H, W, _ptr(pts, c_f32p),
                                            len(pts), int(has_frames), int(has_r), nthreads, ctypes.byref(h)))
    return _table(h)


def link(fyx, search_range, memory=0):
    fyx = _f32(fyx).reshape(-1, 3)
    out = np.empty(len(fyx), np.int64)
    _check(lib().oracle_link(_ptr(fyx, c_f32p), len(fyx), search_range, memory, _ptr(out, c_i64p)))
    return out


def connect(fyx1, fyx2, search_range):
    a, b = _f32(fyx1).reshape(-1, 3), _f32(fyx2).reshape(-1, 3)
    o1 = np.empty(len(a), np.int64)
    o2 = np.empty(len(b), np.int64)
    _check(lib().oracle_connect(_ptr(a, c_f32p), len(a), _ptr(b, c_f32p), len(b), search_range,
                                _ptr(o1, c_i64p), _ptr(o2, c_i64p)))
    return o1, o2


# ---------------------------------------------------- reference shaders (CPU)
def ref_preprocess(p, frame):
    frame = _f32(frame)
    H, W = frame.shape
    out = np.empty_like(frame)
    ref().ref_preprocess(gpu_params(p, H, W), p.truncate_preprocessed, _ptr(frame, c_f32p), _ptr(out, c_f32p))
    return out


def ref_candidates(p, processed, pic_std=0.0):
    processed = _f32(processed)
    H, W = processed.shape
    cap = H * W
    uv = np.empty((cap, 2), np.int32)
    n = ref().ref_candidates(gpu_params(p, H, W), _ptr(processed, c_f32p), pic_std, _ptr(uv, c_i32p), cap)
    return uv[:n].copy()


def ref_walk(p, processed, raw, uv, r=-1.0, characterize=True, pic_std=0.0):
    processed, raw = _f32(processed), _f32(raw)
    H, W = processed.shape
    uv = np.ascontiguousarray(uv, np.int32)
    rows = np.zeros((max(len(uv), 1), 10), np.float32)
    n = ref().ref_walk(gpu_params(p, H, W), _ptr(processed, c_f32p), _ptr(raw, c_f32p), _ptr(uv, c_i32p),
                       len(uv), r, pic_std, int(characterize), _ptr(rows, c_f32p))
    return rows[:n].copy()


def ref_frame_std(frame, divisor=None, temp=None):
    """StdArray::execute with the reference's shaders; temp (2N floats) persists like its buffer."""
    frame = _f32(frame).ravel()
    if temp is None:
        temp = np.zeros(2 * frame.size, np.float32)
    return np.float32(ref().ref_frame_std(_ptr(frame, c_f32p), frame.size,
                                          frame.size if divisor is None else divisor, _ptr(temp, c_f32p)))


def ref_adaptive(p, frame, rows, n_iter, std0, recompute=True):
    frame = _f32(frame).copy()
    H, W = frame.shape
    rows = _f32(rows).reshape(-1, 10)
    temp = np.zeros(2 * H * W, np.float32)
    out = np.zeros((max(len(rows), 1), 10), np.float32)
    n = ref().ref_adaptive(gpu_params(p, H, W), _ptr(frame, c_f32p), _ptr(rows, c_f32p), len(rows), n_iter, std0,
                           int(recompute), _ptr(temp, c_f32p), _ptr(out, c_f32p))
    return out[:n].copy()


def ref_characterize_points(p, processed, raw, yxr):
    processed, raw = _f32(processed), _f32(raw)
    H, W = processed.shape
    rows = np.zeros((max(len(yxr), 1), 10), np.float32)
    yxr = np.asarray(yxr, np.float32)
    rows[: len(yxr), 0] = yxr[:, 0]
    rows[: len(yxr), 1] = yxr[:, 1]
    if yxr.shape[1] > 2:
        rows[: len(yxr), 3] = yxr[:, 2]
    ref().ref_characterize_points(gpu_params(p, H, W), _ptr(processed, c_f32p), _ptr(raw, c_f32p),
                                  _ptr(rows, c_f32p), len(yxr))
    return rows[: len(yxr)].copy()


def ref_laplace(p, frame, sigma):
    frame = _f32(frame)
    H, W = frame.shape
    out = np.empty_like(frame)
    ref().ref_laplace(gpu_params(p, H, W), _ptr(frame, c_f32p), sigma, _ptr(out, c_f32p))
    return out


def ref_logspace_max(p, bottom, middle, top, processed, edge, radius, pic_std=0.0):
    bottom, middle, top, processed = (_f32(a) for a in (bottom, middle, top, processed))
    H, W = middle.shape
    cap = H * W
    uv = np.empty((cap, 2), np.int32)
    n = ref().ref_logspace_max(gpu_params(p, H, W), _ptr(bottom, c_f32p), _ptr(middle, c_f32p), _ptr(top, c_f32p),
                               _ptr(processed, c_f32p), pic_std, edge, radius, _ptr(uv, c_i32p), cap)
    return uv[:n].copy()


def ref_illumination(p, profile, sigma, frame):
    """Smoothed profile and the corrected frame, with the reference's shaders."""
    profile, frame = _f32(profile), _f32(frame).copy()
    H, W = frame.shape
    out = np.empty_like(profile)
    ref().ref_illumination(gpu_params(p, H, W), _ptr(profile, c_f32p), sigma, _ptr(frame, c_f32p), _ptr(out, c_f32p))
    return out, frame
