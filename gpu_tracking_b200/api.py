"""Python API of the B200 engine — the reference's ``gpu_tracking`` functions.

``batch``, ``LoG``, ``characterize_points``, ``link``, ``connect``, ``load`` and
``mean_from_file`` keep the names, arguments, defaults, output columns and
exceptions of the reference (python/gpu_tracking/generated.py:2-227,
python/gpu_tracking/lib.py:74-186, defaults from
gpu_tracking_macros/src/lib.rs:175-683).  Inputs may be numpy arrays, paths
to ``.npy`` files, or CUDA tensors (``data_ptr()`` on the engine's device,
used in place without a copy).

Deliberate differences, each a fix of a reference defect:
  * a 2-D array is one frame (the reference's ``np.atleast_3d`` turns a
    (Y, X) image into Y frames of shape (X, 1));
  * ``characterize_points`` calls the characterization entry point (the shipped
    wrapper calls a non-existent ``characterize_rust``); ``LoG`` forwards its
    radii (the wrapper uses undefined names); ``link`` converts with
    ``astype`` (the wrapper calls ``as_type``).
"""
import ctypes
import os
import threading
import time

import numpy as np

from . import _ffi
from ._params import (COLUMN_INDEX, DTYPE_F32, DTYPE_U8, DTYPE_U16, column_names, log_params, trackpy_params)

__all__ = ["batch", "LoG", "characterize_points", "link", "connect", "load", "mean_from_file"]

_DEVICE = int(os.environ.get("GT_DEVICE", "0"))


def _pandas():
    import pandas as pd
    return pd


class _Frames:
    """A (T, H, W) video as the C ABI sees it: pointer, dtype code, shape."""

    def __init__(self, obj, frames=None, channel=None):
        self.keep = None
        self.frame_numbers = None
        if isinstance(obj, (str, os.PathLike)):
            if os.path.splitext(os.fspath(obj))[1].lower() in _VIDEO_EXT:
                # decoded in the file's own dtype (u8/u16 stay integers),
                # on the GPU straight into device memory where one is usable
                obj = _read_video(obj, frames, channel, device=_gpu_decode())
                if frames is not None:
                    self.frame_numbers = np.asarray([int(k) for k in frames], np.int64)
                    frames = None
            else:
                obj = load(obj)
        if hasattr(obj, "data_ptr") and hasattr(obj, "is_cuda") and obj.is_cuda:
            self._from_tensor(obj, frames)
            return
        arr = np.asarray(obj)
        if arr.ndim == 2:
            arr = arr[None]
        if arr.ndim != 3:
            raise ValueError("expected a (T, Y, X) video, got shape %s" % (arr.shape,))
        if frames is not None:
            keys = [int(k) for k in frames]
            arr = arr[keys]
            self.frame_numbers = np.asarray(keys, np.int64)
        if arr.dtype == np.uint16:
            code = DTYPE_U16
        elif arr.dtype == np.uint8:
            code = DTYPE_U8
        else:
            arr = arr.astype(np.float32, copy=False)
            code = DTYPE_F32
        arr = np.ascontiguousarray(arr)
        self.keep = arr
        self.ptr = ctypes.c_void_p(arr.ctypes.data)
        self.dtype = code
        self.T, self.H, self.W = arr.shape

    def _from_tensor(self, t, frames):
        import torch
        if t.dim() == 2:
            t = t.unsqueeze(0)
        if frames is not None:
            keys = [int(k) for k in frames]
            t = t[keys]
            self.frame_numbers = np.asarray(keys, np.int64)
        t = t.contiguous()
        # the engine's streams do not wait for torch's: the tensor must be
        # complete before its pointer is handed over
        torch.cuda.current_stream(t.device).synchronize()
        if t.dtype == torch.uint16:
            code = DTYPE_U16
        elif t.dtype == torch.uint8:
            code = DTYPE_U8
        else:
            t = t.float().contiguous()
            code = DTYPE_F32
        self.keep = t
        self.ptr = ctypes.c_void_p(t.data_ptr())
        self.dtype = code
        self.T, self.H, self.W = t.shape


def _run(ctx, fn, show_progress):
    """Run a blocking library call on a worker thread; Ctrl-C interrupts it
    cooperatively (the reference's ScopedProgressFuture, macros lib.rs:75-129)."""
    result = {}

    def work():
        result["status"] = fn()

    ctx.interrupt(False)
    th = threading.Thread(target=work, daemon=True)
    th.start()
    bar = None
    try:
        while th.is_alive():
            th.join(0.05)
            if show_progress:
                done, total = ctx.progress()
                if bar is None and total > 0:
                    try:
                        from tqdm import tqdm
                        bar = tqdm(total=total)
                    except Exception:
                        show_progress = False
                if bar is not None:
                    bar.n = done
                    bar.refresh()
    except KeyboardInterrupt:
        ctx.interrupt(True)
        th.join()
        raise
    finally:
        if bar is not None:
            bar.close()
    return result["status"]


def _table_to_frame(ctx, handle, params, has_r=None):
    L = _ffi.lib()
    try:
        n = L.gt_table_nrows(handle)
        cols = column_names(params)
        if has_r is not None and not has_r:
            cols = [c for c in cols if c[0] != "r"]
        # the DataFrame's own dtypes (int64 / float64) filled by one library
        # call; the frame takes the arrays as they are, without a copy
        data = {name: np.empty(n, np.int64 if ty == "int" else np.float64) for name, ty in cols}
        if n and cols:
            idx = (ctypes.c_int32 * len(cols))(*[COLUMN_INDEX[name] for name, _ in cols])
            ptrs = (ctypes.c_void_p * len(cols))(*[data[name].ctypes.data for name, _ in cols])
            ctx.check(L.gt_table_export(handle, idx, len(cols), ptrs))
    finally:
        L.gt_table_free(handle)
    pd = _pandas()
    return pd.DataFrame(data, columns=[c[0] for c in cols], copy=False)


def _locate(video, params, kw):
    ctx = _ffi.context(_DEVICE)
    fr = _Frames(video, kw.get("frames"), kw.get("channel"))
    fn = None
    if fr.frame_numbers is not None:
        fn = fr.frame_numbers
    reset = kw.get("linker_reset_points")
    reset_arr = np.asarray(list(reset) if reset is not None else [], np.int64)
    out = ctypes.c_void_p()
    P64 = ctypes.POINTER(ctypes.c_int64)

    def call():
        return _ffi.lib().gt_batch(ctx.handle, ctypes.byref(params), fr.ptr, fr.dtype, fr.T, fr.H, fr.W,
                                   fn.ctypes.data_as(P64) if fn is not None else None,
                                   reset_arr.ctypes.data_as(P64) if len(reset_arr) else None, len(reset_arr),
                                   ctypes.byref(out))

    st = _run(ctx, call, bool(kw.get("tqdm", True)) and fr.T > 1)
    ctx.check(st)
    return _table_to_frame(ctx, out, params)


def batch(file_or_array, diameter, **kwargs):
    """Trackpy-like (Crocker–Grier) tracking on a B200 GPU.

    Same arguments and defaults as the reference's ``gpu_tracking.batch``
    (python/gpu_tracking/generated.py:2-57): ``separation`` (diameter + 1),
    ``filter_close`` (True), ``noise_size`` (1.0), ``smoothing_size``
    (diameter), ``minmass`` (0), ``max_iterations`` (10), ``characterize``
    (True), ``search_range`` (None: no linking), ``memory`` (0),
    ``doughnut_correction`` (True), ``bg_radius``, ``gap_radius``,
    ``truncate_preprocessed`` (True), ``shift_threshold`` (0.6),
    ``linker_reset_points``, ``frames``, ``tqdm`` (True).  Returns a
    DataFrame with columns frame, y, x, mass[, Rg, raw, signal, ecc]
    [, raw_mass, raw_bg_median, raw_mass_corrected][, particle, duration].
    """
    params = trackpy_params(diameter, **kwargs)
    return _locate(file_or_array, params, kwargs)


def batch_videos(videos, diameter, **kwargs):
    """``batch`` over many videos (any frame sizes and lengths) in one call.

    Returns one DataFrame per video, each equal to ``batch(video, diameter,
    **kwargs)``.  The frames of all videos are located together in waves:
    one launch per stage covers every frame of a wave whatever its size (a
    persistent tile kernel, replayed as a CUDA graph, with the tile height
    and wave size picked by an autotuner); parameter sets the waves do not
    cover (snr, adaptive background, illumination correction) locate video
    by video.  The videos are then linked together in one GPU launch (one
    linker per video running side by side).  ``frames`` and
    ``linker_reset_points`` are not supported here.  Not part of the
    reference's API (it processes one video per call).
    """
    for k in ("frames", "linker_reset_points"):
        if kwargs.get(k) is not None:
            raise TypeError("batch_videos does not take %r" % k)
    params = trackpy_params(diameter, **kwargs)
    ctx = _ffi.context(_DEVICE)
    frs = [_Frames(v) for v in videos]
    if len({f.dtype for f in frs}) > 1:
        frs = [_Frames(np.asarray(v, np.float32)) if not hasattr(v, "is_cuda") else _Frames(v.float())
               for v in videos]
    n = len(frs)
    if n == 0:
        return []
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    ptrs = (vp * n)(*[f.ptr for f in frs])
    Ts = (i64 * n)(*[f.T for f in frs])
    Hs = (i32 * n)(*[f.H for f in frs])
    Ws = (i32 * n)(*[f.W for f in frs])
    outs = (vp * n)()

    def call():
        return _ffi.lib().gt_batch_videos(ctx.handle, ctypes.byref(params), n, ptrs, frs[0].dtype, Ts, Hs, Ws, outs)

    st = _run(ctx, call, False)
    ctx.check(st)
    return [_table_to_frame(ctx, ctypes.c_void_p(outs[i]), params) for i in range(n)]


def LoG(file_or_array, min_radius, max_radius, **kwargs):
    """Laplacian-of-Gaussian blob tracking (generated.py:164-227).

    Adds ``n_radii`` (10), ``log_spacing`` (False) and ``overlap_threshold`` (0)
    to the common arguments; the output includes the detected radius ``r``.
    """
    params = log_params(min_radius, max_radius, **kwargs)
    return _locate(file_or_array, params, kwargs)


def characterize_points(file_or_array, points_to_characterize, diameter=None, **kwargs):
    """Characterize given points as if they had been detected (generated.py:59-162)."""
    has_frames = kwargs.pop("has_frames", None)
    has_r = kwargs.pop("has_r", None)
    pd = _pandas()
    if isinstance(points_to_characterize, pd.DataFrame):
        cols = ["y", "x"]
        if "frame" in points_to_characterize.columns:
            cols = ["frame"] + cols
            if has_frames is None:
                has_frames = True
        if "r" in points_to_characterize.columns:
            cols = cols + ["r"]
            if has_r is None:
                has_r = True
        has_frames = bool(has_frames)
        has_r = bool(has_r)
        points_arr = points_to_characterize[cols].to_numpy().astype("float32")
    else:
        points_arr = np.asarray(points_to_characterize, np.float32)
        has_frames = bool(has_frames)
        has_r = bool(has_r)
    ncols = 2 + int(has_frames) + int(has_r)
    if points_arr.ndim != 2 or points_arr.shape[1] != ncols:
        raise ValueError("unsupported characterize array dimensions.\naccepted dimensions: (Nx2) or (Nx3). "
                         "received: %s" % (list(points_arr.shape),))
    if diameter is None:
        if has_r:
            diameter = 2 * int(points_arr[:, -1].max() + 0.5) + 1
        else:
            raise ValueError("Diameter needs to be specified if the supplied points don't have associated radiuses")
    params = trackpy_params(diameter, **kwargs)
    params.characterize = 1
    params.filter_close = 0
    if has_r:
        params.include_r_in_output = 1
    ctx = _ffi.context(_DEVICE)
    fr = _Frames(file_or_array, kwargs.get("frames"))
    pts = np.ascontiguousarray(points_arr, np.float32)
    out = ctypes.c_void_p()

    def call():
        return _ffi.lib().gt_characterize_points(ctx.handle, ctypes.byref(params), fr.ptr, fr.dtype, fr.T, fr.H,
                                                 fr.W, pts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                 len(pts), int(has_frames), int(has_r), ctypes.byref(out))

    ctx.check(_run(ctx, call, bool(kwargs.get("tqdm", True)) and fr.T > 1))
    return _table_to_frame(ctx, out, params)


def link(to_link, search_range, memory=0):
    """Optimal subnet linking of detections (python/gpu_tracking/lib.py:74-106)."""
    pd = _pandas()
    if isinstance(to_link, pd.DataFrame):
        to_link_np = to_link[["frame", "y", "x"]].to_numpy()
    else:
        to_link_np = to_link
    arr = np.ascontiguousarray(np.asarray(to_link_np).astype("float32"))
    if arr.ndim != 2 or arr.shape[1] != 3:
        raise ValueError("link expects (N, 3) rows of frame, y, x")
    ctx = _ffi.context(_DEVICE)
    ids = np.empty(len(arr), np.int64)
    ctx.check(_ffi.lib().gt_link(ctx.handle, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(arr),
                                 float(search_range), int(memory or 0),
                                 ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
    if isinstance(to_link, pd.DataFrame):
        output = to_link.copy()
        output["particle"] = ids
        return output
    return ids


def connect(to_link1, to_link2, search_range, merge=True):
    """Frame-by-frame association of two detection sets (lib.py:108-158)."""
    pd = _pandas()
    a1 = to_link1[["frame", "y", "x"]].to_numpy() if isinstance(to_link1, pd.DataFrame) else to_link1
    a2 = to_link2[["frame", "y", "x"]].to_numpy() if isinstance(to_link2, pd.DataFrame) else to_link2
    a1 = np.ascontiguousarray(np.asarray(a1).astype("float32"))
    a2 = np.ascontiguousarray(np.asarray(a2).astype("float32"))
    ctx = _ffi.context(_DEVICE)
    r1 = np.empty(len(a1), np.int64)
    r2 = np.empty(len(a2), np.int64)
    FP, IP = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int64)
    ctx.check(_ffi.lib().gt_connect(ctx.handle, a1.ctypes.data_as(FP), len(a1), a2.ctypes.data_as(FP), len(a2),
                                    float(search_range), r1.ctypes.data_as(IP), r2.ctypes.data_as(IP)))
    if isinstance(to_link1, pd.DataFrame):
        output1 = to_link1.copy()
        output1["connect particle"] = r1
    else:
        output1 = r1
    if isinstance(to_link2, pd.DataFrame):
        output2 = to_link2.copy()
        output2["connect particle"] = r2
    else:
        output2 = r2
    if not merge:
        return output1, output2
    return output1.merge(output2, how="outer", on="connect particle")


_VIDEO_EXT = (".tif", ".tiff", ".ets", ".vsi")


def _gpu_decode():
    """Video files decode on the GPU unless GT_DECODE=host or no CUDA device
    is usable from torch."""
    if os.environ.get("GT_DECODE", "device") == "host":
        return False
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def _read_video(path, frames=None, channel=None, as_float=False, device=False):
    """Decode a .tif/.tiff/.ets/.vsi video with the engine's frame providers;
    (T, Y, X) in the file's dtype, or float32: a numpy array decoded on the
    host, or (device=True) a CUDA tensor decoded on the GPU."""
    L = _ffi.lib()
    h = ctypes.c_void_p()
    st = L.gt_video_open(os.fsencode(os.fspath(path)), int(channel or 0), ctypes.byref(h))
    if st != _ffi.GT_OK:
        raise _ffi.to_exception(st, L.gt_video_last_error().decode())
    try:
        T, H, W, dt = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        L.gt_video_info(h, ctypes.byref(T), ctypes.byref(H), ctypes.byref(W), ctypes.byref(dt))
        keys = None if frames is None else np.ascontiguousarray([int(k) for k in frames], np.int64)
        n = T.value if keys is None else len(keys)
        code = DTYPE_F32 if as_float else dt.value
        if device:
            import torch
            ctx = _ffi.context(_DEVICE)
            t_dtype = {DTYPE_U16: torch.uint16, DTYPE_U8: torch.uint8, DTYPE_F32: torch.float32}[code]
            out = torch.empty((n, H.value, W.value), dtype=t_dtype, device="cuda:%d" % _DEVICE)
            torch.cuda.current_stream(out.device).synchronize()
            st = L.gt_video_read_device(ctx.handle, h,
                                        keys.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)) if keys is not None
                                        else None, n, code, ctypes.c_void_p(out.data_ptr()))
            if st != _ffi.GT_OK:
                raise _ffi.to_exception(st, L.gt_video_last_error().decode())
            return out
        np_dtype = {DTYPE_U16: np.uint16, DTYPE_U8: np.uint8, DTYPE_F32: np.float32}[code]
        out = np.empty((n, H.value, W.value), np_dtype)
        st = L.gt_video_read(h, keys.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)) if keys is not None else None,
                             n, code, ctypes.c_void_p(out.ctypes.data))
        if st != _ffi.GT_OK:
            raise _ffi.to_exception(st, L.gt_video_last_error().decode())
        return out
    finally:
        L.gt_video_close(h)


def load(path, frames=None, channel=None):
    """Load a video as a (T, Y, X) float32 array (lib.py:174-186, load_rust
    python_bindings.rs:223-270).

    .tif/.tiff stacks and Olympus .ets/.vsi files (``channel``, default 0)
    are decoded by the engine's frame providers; ``.npy`` files are read with
    numpy (kept in their dtype).  ``frames`` selects frame indices.
    """
    path = os.fspath(path)
    ext = os.path.splitext(path)[1].lower()
    if ext == "":
        raise ValueError("could not determine extension of file '%s'" % path)
    if ext not in (".npy",) + _VIDEO_EXT:
        raise ValueError("unsupported file format: %s" % ext.lstrip("."))
    if ext != ".vsi" and not os.path.exists(path):
        raise FileNotFoundError("could not find file '%s'" % path)
    if ext in _VIDEO_EXT:
        return _read_video(path, frames, channel, as_float=True)
    arr = np.load(path, mmap_mode="r")
    if arr.ndim == 2:
        arr = arr[None]
    if frames is not None:
        arr = arr[[int(k) for k in frames]]
    return np.ascontiguousarray(arr)


def mean_from_file(path, channel=None):
    """Mean frame of a video file (lib.py:161-172), computed on the GPU."""
    fr = _Frames(path, None, channel)
    ctx = _ffi.context(_DEVICE)
    out = np.empty((fr.H, fr.W), np.float32)
    ctx.check(_ffi.lib().gt_mean_frame(ctx.handle, fr.ptr, fr.dtype, fr.T, fr.H, fr.W,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    return out
