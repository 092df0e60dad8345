"""ctypes binding of libgt_b200.so (the C ABI of include/gpu_tracking_b200.h).

The library is built in-tree by ``gpu_tracking_b200.build``.  There is no
fallback: if the CUDA library cannot be loaded or no CUDA device is present,
every call raises.
"""
import ctypes
import os
import threading

from ._params import GtParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgt_b200.so")

GT_OK = 0
STATUS_NAMES = {
    1: "InvalidArgument", 2: "DimensionMismatch", 3: "EmptyIterator", 4: "NonSortedCharacterization",
    5: "FrameOutOfBounds", 6: "NonStandardArrayLayout", 7: "ArrayDimensionsError", 8: "TooDenseToLink",
    9: "Interrupted", 10: "CapacityExceeded", 11: "CudaError", 12: "NoDevice", 13: "SubnetTooExpensive",
    14: "Internal", 15: "FileNotFound", 16: "ReadError",
}

_lib = None
_lock = threading.Lock()


class GpuTrackingError(RuntimeError):
    """Raised for CUDA or internal failures of the engine."""

    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


def to_exception(status, message):
    """Map a gt_status to the exception the reference raises
    (gpu_tracking_python/src/python_bindings.rs:160-193)."""
    if status == 9:
        return KeyboardInterrupt(message)
    if status == 12:
        return ConnectionError(message)
    if status == 15:
        return FileNotFoundError(message)
    if status == 16:
        return ValueError(message)
    if status in (1, 2, 3, 4, 5, 6, 7, 8, 10):
        return ValueError(message)
    return GpuTrackingError(status, message)


class TrainOpts(ctypes.Structure):
    """gt_train_opts (include/gpu_tracking_b200.h)."""
    _fields_ = [("steps", ctypes.c_int32), ("batch", ctypes.c_int32), ("crop", ctypes.c_int32),
                ("lr", ctypes.c_float), ("pos_weight", ctypes.c_float), ("offset_weight", ctypes.c_float),
                ("seed", ctypes.c_uint32)]


def lib():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        P = ctypes.POINTER
        L.gt_version.restype = ctypes.c_char_p
        L.gt_params_default.argtypes = [P(GtParams)]
        L.gt_create.argtypes = [i32, P(vp)]
        L.gt_destroy.argtypes = [vp]
        L.gt_last_error.argtypes = [vp]
        L.gt_last_error.restype = ctypes.c_char_p
        L.gt_set_interrupt.argtypes = [vp, P(i32)]
        L.gt_progress.argtypes = [vp, P(i64), P(i64)]
        L.gt_table_nrows.argtypes = [vp]
        L.gt_table_nrows.restype = i64
        L.gt_table_column_f32.argtypes = [vp, i32, P(f32)]
        L.gt_table_column_i64.argtypes = [vp, i32, P(i64)]
        L.gt_table_export.argtypes = [vp, P(i32), i32, P(vp)]
        L.gt_table_has_column.argtypes = [vp, i32]
        L.gt_table_has_column.restype = i32
        L.gt_table_free.argtypes = [vp]
        L.gt_batch.argtypes = [vp, P(GtParams), vp, i32, i64, i32, i32, P(i64), P(i64), i64, P(vp)]
        L.gt_batch_videos.argtypes = [vp, P(GtParams), i32, P(vp), i32, P(i64), P(i32), P(i32), P(vp)]
        L.gt_characterize_points.argtypes = [vp, P(GtParams), vp, i32, i64, i32, i32, P(f32), i64, i32, i32,
                                             P(vp)]
        L.gt_link.argtypes = [vp, P(f32), i64, f32, ctypes.c_uint32, P(i64)]
        L.gt_connect.argtypes = [vp, P(f32), i64, P(f32), i64, f32, P(i64), P(i64)]
        L.gt_mean_frame.argtypes = [vp, vp, i32, i64, i32, i32, P(f32)]
        L.gt_profile_enable.argtypes = [vp, i32]
        L.gt_profile_read.argtypes = [vp, ctypes.c_char_p, P(i64), P(ctypes.c_double)]
        L.gt_launch_count.argtypes = [vp]
        L.gt_launch_count.restype = i64
        L.gt_train_opts_default.argtypes = [P(TrainOpts)]
        L.gt_proposal_num_params.restype = i64
        L.gt_proposal_create.argtypes = [vp, ctypes.c_uint64, P(vp)]
        L.gt_proposal_destroy.argtypes = [vp]
        L.gt_proposal_set.argtypes = [vp, vp, P(f32), f32, f32, f32]
        L.gt_proposal_get.argtypes = [vp, vp, P(f32), P(f32), P(f32), P(f32)]
        L.gt_proposal_train.argtypes = [vp, vp, vp, i32, i64, i32, i32, P(i64), P(f32), P(f32), i64, P(TrainOpts),
                                        P(f32)]
        L.gt_proposal_maps.argtypes = [vp, vp, vp, i32, i64, i32, i32, P(f32)]
        L.gt_batch_learned.argtypes = [vp, P(GtParams), vp, vp, i32, i64, i32, i32, P(i64), P(i64), i64, P(vp)]
        L.gt_video_open.argtypes = [ctypes.c_char_p, i32, P(vp)]
        L.gt_video_open.restype = i32
        L.gt_video_info.argtypes = [vp, P(i64), P(i32), P(i32), P(i32)]
        L.gt_video_info.restype = i32
        L.gt_video_read.argtypes = [vp, P(i64), i64, i32, vp]
        L.gt_video_read.restype = i32
        L.gt_video_read_device.argtypes = [vp, vp, P(i64), i64, i32, vp]
        L.gt_video_read_device.restype = i32
        L.gt_video_close.argtypes = [vp]
        L.gt_video_last_error.restype = ctypes.c_char_p
        L.gt_last_walk_starts.argtypes = [vp]
        L.gt_last_walk_starts.restype = i64
        L.gt__proposal_loss_grad.argtypes = [vp, vp, vp, i32, i64, i32, i32, P(i64), P(f32), P(f32), i64, P(i32), i32,
                                             i32, f32, f32, P(f32), P(f32)]
        for name in ("gt_create", "gt_set_interrupt", "gt_progress", "gt_table_column_f32", "gt_table_column_i64",
                     "gt_table_export", "gt_batch", "gt_batch_videos", "gt_characterize_points", "gt_link", "gt_connect", "gt_mean_frame",
                     "gt_profile_enable", "gt_profile_read", "gt_proposal_create", "gt_proposal_set",
                     "gt_proposal_get", "gt_proposal_train", "gt_proposal_maps", "gt_batch_learned",
                     "gt__proposal_loss_grad"):
            getattr(L, name).restype = i32
        _lib = L
        return L


class Context:
    """One engine context (device, streams, persistent device buffers)."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        st = lib().gt_create(int(device), ctypes.byref(self._h))
        if st != GT_OK:
            raise to_exception(st, "could not create a context on CUDA device %d" % device)
        self.device = device
        self._flag = ctypes.c_int32(0)
        lib().gt_set_interrupt(self._h, ctypes.byref(self._flag))

    @property
    def handle(self):
        return self._h

    def check(self, st):
        if st != GT_OK:
            msg = lib().gt_last_error(self._h)
            raise to_exception(st, msg.decode() if msg else "")

    def interrupt(self, on=True):
        self._flag.value = 1 if on else 0

    def progress(self):
        d, t = ctypes.c_int64(), ctypes.c_int64()
        lib().gt_progress(self._h, ctypes.byref(d), ctypes.byref(t))
        return d.value, t.value

    def profile(self, enable=True):
        self.check(lib().gt_profile_enable(self._h, 1 if enable else 0))

    def profile_read(self, name):
        n, ms = ctypes.c_int64(), ctypes.c_double()
        self.check(lib().gt_profile_read(self._h, name.encode(), ctypes.byref(n), ctypes.byref(ms)))
        return n.value, ms.value

    def launch_count(self):
        return lib().gt_launch_count(self._h)

    def close(self):
        if self._h:
            lib().gt_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def context(device=0):
    """The process-wide context of a device (created on first use)."""
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[device] = ctx
    return ctx
