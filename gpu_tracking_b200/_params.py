"""Tracking parameters: the Python mirror of the reference's TrackingParams.

The field layout matches ``gt_params`` in ``include/gpu_tracking_b200.h``.
Defaults are the ones the reference's Python functions apply
(gpu_tracking_macros/src/lib.rs:187-683), which differ from
``TrackingParams::default()`` (src/gpu_setup.rs:61-97) — e.g. the Python
layer defaults to ``characterize=True`` and ``doughnut_correction=True``.
"""
import ctypes

STYLE_TRACKPY = 0
STYLE_LOG = 1

DTYPE_U16 = 0
DTYPE_F32 = 1
DTYPE_U8 = 2


class GtParams(ctypes.Structure):
    _fields_ = [
        ("style", ctypes.c_int32),
        ("diameter", ctypes.c_uint32),
        ("separation", ctypes.c_uint32),
        ("filter_close", ctypes.c_int32),
        ("min_radius", ctypes.c_float),
        ("max_radius", ctypes.c_float),
        ("n_radii", ctypes.c_uint32),
        ("log_spacing", ctypes.c_int32),
        ("overlap_threshold", ctypes.c_float),
        ("minmass", ctypes.c_float),
        ("max_iterations", ctypes.c_uint32),
        ("characterize", ctypes.c_int32),
        ("has_search_range", ctypes.c_int32),
        ("search_range", ctypes.c_float),
        ("memory", ctypes.c_uint32),
        ("doughnut_correction", ctypes.c_int32),
        ("has_bg_radius", ctypes.c_int32),
        ("bg_radius", ctypes.c_float),
        ("has_gap_radius", ctypes.c_int32),
        ("gap_radius", ctypes.c_float),
        ("has_snr", ctypes.c_int32),
        ("snr", ctypes.c_float),
        ("has_minmass_snr", ctypes.c_int32),
        ("minmass_snr", ctypes.c_float),
        ("truncate_preprocessed", ctypes.c_int32),
        ("has_illumination_sigma", ctypes.c_int32),
        ("illumination_sigma", ctypes.c_float),
        ("illumination_correction_per_frame", ctypes.c_int32),
        ("has_adaptive_background", ctypes.c_int32),
        ("adaptive_background", ctypes.c_uint32),
        ("include_r_in_output", ctypes.c_int32),
        ("shift_threshold", ctypes.c_float),
        ("noise_size", ctypes.c_float),
        ("has_smoothing_size", ctypes.c_int32),
        ("smoothing_size", ctypes.c_uint32),
    ]


# Keyword arguments the reference's trackpy-style signature accepts but never
# reads (ParamStyle::Trackpy fields maxsize, threshold, invert, percentile,
# topn, preprocess; gpu_tracking_macros/src/lib.rs:487-569).
IGNORED_TRACKPY_KWARGS = ("maxsize", "threshold", "invert", "percentile", "topn", "preprocess")

COMMON_KWARGS = (
    "noise_size", "smoothing_size", "minmass", "max_iterations", "characterize", "search_range",
    "memory", "doughnut_correction", "bg_radius", "gap_radius", "snr", "minmass_snr",
    "truncate_preprocessed", "correct_illumination", "illumination_sigma",
    "illumination_correction_per_frame", "adaptive_background", "shift_threshold",
    "linker_reset_points", "frames", "tqdm", "channel",
)
TRACKPY_KWARGS = COMMON_KWARGS + ("separation", "filter_close") + IGNORED_TRACKPY_KWARGS
LOG_KWARGS = COMMON_KWARGS + ("n_radii", "log_spacing", "overlap_threshold")


def _opt(p, name, value, conv=float):
    if value is None:
        setattr(p, "has_" + name, 0)
        setattr(p, name, 0)
    else:
        setattr(p, "has_" + name, 1)
        setattr(p, name, conv(value))


def _common(p, kw):
    """Common arguments with the Python-layer defaults (macros lib.rs:175-481)."""
    p.noise_size = float(kw.get("noise_size") if kw.get("noise_size") is not None else 1.0)
    ss = kw.get("smoothing_size")
    _opt(p, "smoothing_size", ss, int)
    mm = kw.get("minmass")
    p.minmass = float(mm if mm is not None else 0.0)
    mi = kw.get("max_iterations")
    p.max_iterations = int(mi if mi is not None else 10)
    ch = kw.get("characterize")
    p.characterize = int(bool(True if ch is None else ch))
    _opt(p, "search_range", kw.get("search_range"))
    mem = kw.get("memory")
    p.memory = int(mem if mem is not None else 0)
    dc = kw.get("doughnut_correction")
    p.doughnut_correction = int(bool(True if dc is None else dc))
    bg = kw.get("bg_radius")
    _opt(p, "bg_radius", bg)
    # gap_radius = bg_radius.map(|_| gap_radius.unwrap_or(0.))  (macros lib.rs:284-291)
    gap = kw.get("gap_radius")
    _opt(p, "gap_radius", None if bg is None else (gap if gap is not None else 0.0))
    _opt(p, "snr", kw.get("snr"))
    _opt(p, "minmass_snr", kw.get("minmass_snr"))
    tp = kw.get("truncate_preprocessed")
    p.truncate_preprocessed = int(bool(True if tp is None else tp))
    isig = kw.get("illumination_sigma")
    if isig is None and kw.get("correct_illumination"):
        isig = 30.0
    _opt(p, "illumination_sigma", isig)
    p.illumination_correction_per_frame = int(bool(kw.get("illumination_correction_per_frame") or False))
    _opt(p, "adaptive_background", kw.get("adaptive_background"), int)
    st = kw.get("shift_threshold")
    p.shift_threshold = float(st if st is not None else 0.6)


def trackpy_params(diameter, **kw):
    """Parameters of ``batch`` (macros lib.rs:487-569)."""
    unknown = set(kw) - set(TRACKPY_KWARGS)
    if unknown:
        raise TypeError("unexpected keyword argument(s): %s" % ", ".join(sorted(unknown)))
    p = GtParams()
    p.style = STYLE_TRACKPY
    p.diameter = int(diameter)
    sep = kw.get("separation")
    p.separation = int(sep if sep is not None else int(diameter) + 1)
    fc = kw.get("filter_close")
    p.filter_close = int(bool(True if fc is None else fc))
    p.include_r_in_output = 0
    p.n_radii = 0
    _common(p, kw)
    return p


def log_params(min_radius, max_radius, **kw):
    """Parameters of ``LoG`` (macros lib.rs:571-639)."""
    unknown = set(kw) - set(LOG_KWARGS)
    if unknown:
        raise TypeError("unexpected keyword argument(s): %s" % ", ".join(sorted(unknown)))
    p = GtParams()
    p.style = STYLE_LOG
    p.min_radius = float(min_radius)
    p.max_radius = float(max_radius)
    nr = kw.get("n_radii")
    p.n_radii = int(nr if nr is not None else 10)
    p.log_spacing = int(bool(kw.get("log_spacing") or False))
    ot = kw.get("overlap_threshold")
    p.overlap_threshold = float(ot if ot is not None else 0.0)
    p.include_r_in_output = 1
    p.diameter = 0
    p.separation = 0
    _common(p, kw)
    return p


def column_names(p):
    """Output columns and pandas dtypes (src/execute_gpu.rs:482-519)."""
    names = [("frame", "int"), ("y", "float"), ("x", "float"), ("mass", "float")]
    if p.include_r_in_output:
        names.append(("r", "float"))
    if p.characterize:
        names += [("Rg", "float"), ("raw", "float"), ("signal", "float"), ("ecc", "float")]
    if p.doughnut_correction:
        names += [("raw_mass", "float"), ("raw_bg_median", "float"), ("raw_mass_corrected", "float")]
    if p.has_search_range:
        names += [("particle", "int"), ("duration", "int")]
    return names


# column name -> gt_column index (include/gpu_tracking_b200.h)
COLUMN_INDEX = {
    "frame": 0, "y": 1, "x": 2, "mass": 3, "r": 4, "Rg": 5, "raw": 6, "signal": 7, "ecc": 8,
    "raw_mass": 9, "raw_bg_median": 10, "raw_mass_corrected": 11, "particle": 12, "duration": 13,
    "max_intensity": 14, "count": 15,
}
NUM_COLUMNS = 16
INT_COLUMNS = ("frame", "particle", "duration")


def derived(p, H, W):
    """gpuparams_from_tracking_params (src/gpu_setup.rs:528-580) as a dict.

    Used by the host library's tests; the CUDA library computes the same
    quantities in C++ (gpu_tracking_b200/csrc/gt_params.cpp).
    """
    import numpy as np
    f32 = np.float32
    if p.style == STYLE_TRACKPY:
        smoothing = p.smoothing_size if p.has_smoothing_size else p.diameter
        dil = int(f32(2.0) * f32(p.separation) / np.sqrt(f32(2.0)))
        b = (p.separation // 2 - 1) % (1 << 32)
        margin = max(p.diameter // 2, b, smoothing // 2)
        if margin >= 1 << 31:
            margin -= 1 << 32
        return dict(smoothing=smoothing, circle=p.diameter, dilation=dil, margin=margin)
    smoothing = p.smoothing_size if p.has_smoothing_size else int(f32(p.max_radius) + f32(0.5)) * 2 + 1
    return dict(smoothing=smoothing, circle=0, dilation=0, margin=0)


__all__ = ["GtParams", "trackpy_params", "log_params", "column_names", "COLUMN_INDEX"]
