"""gt_link_noalloc: linking with no device allocation, through the C ABI.

Some callers cannot allocate device memory while they run: a live acquisition
loop that links each batch of detections as frames arrive (cudaMalloc and
cudaFree synchronise the whole device and would stall it), or a process whose
device memory belongs to another allocator.  gt_link_noalloc serves them from
one static device array.  This test calls it twice in a row on device-resident
detections and checks that its particle ids equal those of the ordinary entry
point (gt_link), exactly — ids are integers, the tolerance is zero.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def detections(seed, T, n, R, size):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, size, (n, 2))
    rows = []
    for t in range(T):
        keep = rng.random(n) > 0.05
        for k in np.flatnonzero(keep):
            rows.append((t, pos[k, 0], pos[k, 1]))
        pos = pos + rng.normal(0, R / 3, pos.shape)
        dead = rng.random(n) < 0.1
        pos[dead] = rng.uniform(0, size, (dead.sum(), 2))
    return np.array(rows, np.float32)


def link_noalloc(ctx, rows, radius, memory):
    import torch

    from gpu_tracking_b200 import _ffi
    L = _ffi.lib()
    L.gt_link_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                  ctypes.c_uint32, ctypes.c_void_p]
    L.gt_link_noalloc.restype = ctypes.c_int32
    d_rows = torch.from_numpy(rows).cuda()
    d_ids = torch.full((len(rows),), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.check(L.gt_link_noalloc(ctx.handle, ctypes.c_void_p(d_rows.data_ptr()), len(rows), float(radius),
                                int(memory), ctypes.c_void_p(d_ids.data_ptr())))
    return d_ids.cpu().numpy()


def test_link_noalloc_matches_link_twice():
    pytest.importorskip("torch")
    import gpu_tracking_b200 as gt
    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    cases = [(detections(11, 40, 120, 5.0, 200.0), 5.0, 3),
             (detections(12, 25, 60, 4.0, 100.0), 4.0, 1)]
    for rows, radius, memory in cases:
        want = gt.link(rows, radius, memory)
        got = link_noalloc(ctx, rows, radius, memory)
        assert np.array_equal(got, want)


def test_link_noalloc_rejects_oversized_input():
    pytest.importorskip("torch")
    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    rows = np.zeros((40000, 3), np.float32)
    with pytest.raises(ValueError):
        link_noalloc(ctx, rows, 2.0, 0)
