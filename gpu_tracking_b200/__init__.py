"""gpu_tracking_b200 — particle locating and linking for NVIDIA B200 (sm_100a).

A drop-in for the hot path of amfaber/gpu_tracking: the same Python calls
(batch, LoG, characterize_points, link, connect, load, mean_from_file) and a
C ABI (include/gpu_tracking_b200.h) backed by hand-written CUDA kernels.
"""
from .api import LoG, batch, batch_videos, characterize_points, connect, link, load, mean_from_file

__all__ = ["batch", "batch_videos", "LoG", "characterize_points", "link", "connect", "load", "mean_from_file"]
__version__ = "0.1.0"
