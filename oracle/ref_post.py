"""The reference's own Rust post-processing and linking, run on the CPU.

TEST INFRASTRUCTURE ONLY (part of the oracle).  oracle/rust2py.py translates
the reference's Rust functions (post_process with filter_close_trackpy,
prune_blobs_log and the doughnut block; Linker, link, linker_all,
connect_all; circle_inds / annulus_inds; column_names and the duration
column) into oracle/_ref/rust_ref.py.  This module drives them the way the
reference's execute_gpu worker thread does (src/execute_gpu.rs:912-994):

  * one Linker when search_range is set (Linker::new(range,
    memory.unwrap_or(0)), src/execute_gpu.rs:917-919);
  * the doughnut kernels of make_kernels (the worker's FloatMemoizer set-up,
    translated from src/execute_gpu.rs:924-938) when doughnut_correction;
  * post_process(results, &mut output, frame_index, linker, kernels,
    frame, dims, params, None) for every frame in order, the frame being the
    raw f32 frame the worker receives when the doughnut correction is on;
  * linker.finish() and the duration column (append_durations, translated
    from src/execute_gpu.rs:1164-1181).

The per-frame detections (the ResultRow records the GPU passes hand to the
worker) come from the reference's WGSL shaders translated by
oracle/wgsl2cpp.py (oracle/_ref/libgt_ref.so), in the shaders' serial
dispatch order.  link() and connect() mirror link_rust / connect_rust
(gpu_tracking_python/src/python_bindings.rs:274-312): FrameSubsetter over
(frame, y, x) rows, then linker_all / connect_all.

Available only where the reference checkout was present when the oracle was
built; the golden vectors in tests/golden/ carry its outputs elsewhere.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_MOD = None


def available():
    return os.path.exists(os.path.join(HERE, "_ref", "rust_ref.py"))


def module():
    global _MOD
    if _MOD is None:
        if HERE not in sys.path:
            sys.path.insert(0, HERE)
        spec = importlib.util.spec_from_file_location("rust_ref", os.path.join(HERE, "_ref", "rust_ref.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _MOD = mod
    return _MOD


def _rt():
    module()
    import rust_rt
    return rust_rt


class TrackingParams:
    """The fields of the reference's TrackingParams (src/gpu_setup.rs:10-59)
    that the post-processing reads, from a gt_params structure."""

    def __init__(self, p, linker_reset_points=None):
        rt = _rt()
        F = np.float32
        if p.style == 0:
            self.style = rt.REnum("Trackpy", (), dict(diameter=int(p.diameter), separation=int(p.separation),
                                                      filter_close=bool(p.filter_close)))
        else:
            self.style = rt.REnum("Log", (), dict(min_radius=F(p.min_radius), max_radius=F(p.max_radius),
                                                  n_radii=int(p.n_radii), log_spacing=bool(p.log_spacing),
                                                  overlap_threshold=F(p.overlap_threshold)))
        self.include_r_in_output = bool(p.include_r_in_output)
        self.characterize = bool(p.characterize)
        self.doughnut_correction = bool(p.doughnut_correction)
        self.search_range = F(p.search_range) if p.has_search_range else None
        self.memory = int(p.memory)
        self.linker_reset_points = list(linker_reset_points) if linker_reset_points is not None else None
        self.bg_radius = F(p.bg_radius) if p.has_bg_radius else None
        self.gap_radius = F(p.gap_radius) if p.has_gap_radius else None


def result_rows(rows):
    """ResultRow records from (n, 10) float32 shader output rows."""
    R = module().ResultRow
    names = [n for n, _ in R._fields]
    return [R(**{n: np.float32(v) for n, v in zip(names, r)}) for r in np.asarray(rows, np.float32)]


def post_process_video(p, frames, rows_per_frame, linker_reset_points=None):
    """The worker thread's loop over the frames' detections; returns the
    output table (rows x columns, float32) and its column names."""
    m = module()
    tp = TrackingParams(p, linker_reset_points)
    linker = m.Linker.new(tp.search_range, tp.memory) if tp.search_range is not None else None
    kernels = m.make_kernels(tp, tp.doughnut_correction)
    output = []
    frames = np.asarray(frames, np.float32)
    T, H, W = frames.shape
    for t in range(T):
        results = result_rows(rows_per_frame[t])
        frame = frames[t].ravel() if tp.doughnut_correction else None
        m.post_process(results, output, t, linker, kernels, frame, [H, W], tp, None)
    part_durations = linker.finish() if linker is not None else None
    output = m.append_durations(output, part_durations, tp)
    names, _ = m.column_names(tp)
    cols = [n for n, _ in names]
    return np.asarray(output, np.float32).reshape(-1, len(cols)), cols


def shader_rows_trackpy(p, frame):
    """The trackpy-style detections of one frame from the reference's
    shaders: preprocess, extract_max candidates, walk + characterize."""
    from . import loader
    f = np.asarray(frame, np.float32)
    proc = loader.ref_preprocess(p, f)
    cands = loader.ref_candidates(p, proc)
    return loader.ref_walk(p, proc, f, cands, characterize=bool(p.characterize))


def shader_rows_log(p, frame):
    """The LoG detections of one frame from the reference's shaders: the
    separable LoG planes of every radius, the scale-space maxima and their
    walks, radius by radius."""
    from . import loader
    f = np.asarray(frame, np.float32)
    radii = loader.log_radii(p)
    proc = loader.ref_preprocess(p, f)
    planes = [loader.ref_laplace(p, f, np.float32(r) / np.sqrt(np.float32(2.0))) for r in radii]
    rows = []
    n = len(radii)
    for i in range(n):
        edge = -1 if i == 0 else (1 if i == n - 1 else 0)
        bottom = planes[i - 1] if i > 0 else np.zeros_like(f)
        top = planes[i + 1] if i < n - 1 else np.zeros_like(f)
        cands = loader.ref_logspace_max(p, bottom, planes[i], top, proc, edge, radii[i])
        rows.append(loader.ref_walk(p, proc, f, cands, r=float(radii[i]), characterize=bool(p.characterize)))
    return np.concatenate(rows) if rows else np.zeros((0, 10), np.float32)


def batch(p, frames, linker_reset_points=None):
    """The whole path with the reference's own code: shaders, then the Rust
    post-processing and linking.  Returns (table, column names)."""
    frames = np.asarray(frames, np.float32)
    fn = shader_rows_log if p.style == 1 else shader_rows_trackpy
    rows = [fn(p, frames[t]) for t in range(len(frames))]
    return post_process_video(p, frames, rows, linker_reset_points)


def _subsetter_iter(fyx):
    m = module()
    arr = np.ascontiguousarray(fyx, np.float32).reshape(-1, 3)
    return m.FrameSubsetter.new(arr, 0, (1, 2), None, m.SubsetterType.Linking).into_linking_iter()


def link(fyx, search_range, memory=0):
    """link_rust: particle ids of (frame, y, x) rows."""
    return np.asarray(module().linker_all(_subsetter_iter(fyx), np.float32(search_range), int(memory)), np.int64)


def connect(fyx1, fyx2, search_range):
    """connect_rust: ids of two detection sets linked frame by frame."""
    r1, r2 = module().connect_all(_subsetter_iter(fyx1), _subsetter_iter(fyx2), np.float32(search_range))
    return np.asarray(r1, np.int64), np.asarray(r2, np.int64)
