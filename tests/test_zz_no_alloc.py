"""gt_link_noalloc: linking with no device allocation, through the C ABI.

Some callers cannot allocate device memory while they run: a live acquisition
loop that links each batch of detections as frames arrive (cudaMalloc and
cudaFree synchronise the whole device and would stall it), or a process whose
device memory belongs to another allocator.  gt_link_noalloc serves them from
one static device array.  These tests call it on device-resident detections
and check its particle ids against the oracle's linker and against the
ordinary entry point (gt_link), exactly — ids are integers, the tolerance is
zero — on two calls in a row, so state left in the shared array by one call
would show in the next.  The device-side frame grouping (which gt_link does
on the host) is covered by inputs that start above frame 0, carry NaN frame
values, are unsorted, or hold a frame larger than the per-frame limit.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def detections(seed, T, n, R, size, first_frame=0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, size, (n, 2))
    rows = []
    for t in range(T):
        keep = rng.random(n) > 0.05
        for k in np.flatnonzero(keep):
            rows.append((first_frame + t, pos[k, 0], pos[k, 1]))
        pos = pos + rng.normal(0, R / 3, pos.shape)
        dead = rng.random(n) < 0.1
        pos[dead] = rng.uniform(0, size, (dead.sum(), 2))
    return np.array(rows, np.float32)


def _fn():
    from gpu_tracking_b200 import _ffi
    L = _ffi.lib()
    L.gt_link_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                  ctypes.c_uint32, ctypes.c_void_p]
    L.gt_link_noalloc.restype = ctypes.c_int32
    return L.gt_link_noalloc


def link_noalloc(ctx, rows, radius, memory):
    import torch
    d_rows = torch.from_numpy(np.ascontiguousarray(rows, np.float32)).cuda()
    d_ids = torch.full((len(rows),), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.check(_fn()(ctx.handle, ctypes.c_void_p(d_rows.data_ptr()), len(rows), float(radius), int(memory),
                    ctypes.c_void_p(d_ids.data_ptr())))
    return d_ids.cpu().numpy()


def test_link_noalloc_matches_oracle_and_link_twice():
    pytest.importorskip("torch")
    import torch

    import gpu_tracking_b200 as gt
    from gpu_tracking_b200 import _ffi
    from oracle import loader
    ctx = _ffi.context(0)
    cases = [(detections(11, 40, 120, 5.0, 200.0), 5.0, 3),
             (detections(12, 25, 60, 4.0, 100.0), 4.0, 1)]
    for rows, radius, memory in cases:
        want = loader.link(rows, radius, memory)
        got = link_noalloc(ctx, rows, radius, memory)
        assert np.array_equal(got, want)
        assert np.array_equal(got, gt.link(rows, radius, memory))
    # the caller's current device is left as it was
    assert torch.cuda.current_device() == 0


def test_link_noalloc_device_grouping_edges():
    pytest.importorskip("torch")
    from gpu_tracking_b200 import _ffi
    from oracle import loader
    ctx = _ffi.context(0)
    # detections that start at frame 5: frames 0..4 form one empty group
    late = detections(21, 12, 40, 4.0, 80.0, first_frame=5)
    # NaN frame values join the group in progress (a NaN is neither above nor
    # below the current frame value)
    nan_rows = detections(22, 10, 40, 4.0, 80.0)
    nan_rows[[7, 50, 51, 200], 0] = np.nan
    for rows in (late, nan_rows):
        want = loader.link(rows, 4.0, 2)
        for _ in range(2):
            assert np.array_equal(link_noalloc(ctx, rows, 4.0, 2), want)


def test_link_noalloc_errors():
    pytest.importorskip("torch")
    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    rows = detections(23, 6, 30, 4.0, 80.0)
    unsorted = rows.copy()
    unsorted[[3, 40]] = unsorted[[40, 3]]
    with pytest.raises(ValueError, match="sorted"):
        link_noalloc(ctx, unsorted, 4.0, 0)
    big = np.zeros((4097, 3), np.float32)
    big[:, 1] = np.arange(4097) % 64 * 9.0
    big[:, 2] = np.arange(4097) // 64 * 9.0
    with pytest.raises(ValueError, match="per frame"):
        link_noalloc(ctx, big, 2.0, 0)
    with pytest.raises(ValueError):
        link_noalloc(ctx, np.zeros((40000, 3), np.float32), 2.0, 0)
    # still usable after the errors
    from oracle import loader
    assert np.array_equal(link_noalloc(ctx, rows, 4.0, 1), loader.link(rows, 4.0, 1))


def _driver_alloc(nbytes):
    """An allocation of exactly nbytes (a multiple of 2 MiB) from the driver,
    so that its address range is the requested size."""
    import torch
    torch.zeros(1, device="cuda")
    cu = ctypes.CDLL("libcuda.so.1")
    ptr = ctypes.c_uint64()
    assert cu.cuMemAlloc_v2(ctypes.byref(ptr), ctypes.c_size_t(nbytes)) == 0
    return cu, ptr.value


def test_link_noalloc_rejects_buffers_shorter_than_n():
    """n larger than the caller's id buffer: the call must stop before any
    kernel runs.  memory = 9 is also beyond the entry point's limit, so even
    without the buffer check no kernel would touch the short buffer; the
    message says which check stopped it."""
    pytest.importorskip("torch")
    import torch

    from gpu_tracking_b200 import _ffi
    ctx = _ffi.context(0)
    n_ids = (2 << 20) // 8
    cu, ids_ptr = _driver_alloc(2 << 20)
    try:
        d_rows = torch.zeros((n_ids + 1, 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        st = _fn()(ctx.handle, ctypes.c_void_p(d_rows.data_ptr()), n_ids + 1, 2.0, 9, ctypes.c_void_p(ids_ptr))
        assert st == 1, st
        assert b"past the end" in _ffi.lib().gt_last_error(ctx.handle)
    finally:
        cu.cuMemFree_v2(ctypes.c_uint64(ids_ptr))
