"""Failure paths, injected from the host (no GPU fault is ever provoked).

* Interrupt: the reference's cooperative Arc<AtomicBool>
  (src/execute_gpu.rs:1094-1099, src/linking.rs:707-711) is the flag passed to
  gt_set_interrupt.  A host thread sets it while a long call runs; the call
  stops at its next chunk boundary with GT_ERR_INTERRUPTED, which the Python
  layer raises as KeyboardInterrupt (python_bindings.rs:160-193), and the
  context stays usable.
* Progress: gt_progress rises monotonically to the call's frame total (the
  reference's progress mutex, src/execute_gpu.rs:972-975).
* Capacity: the reference truncates candidates and results at fixed buffer
  sizes (src/gpu_setup.rs:208-215,246-253); the engine's kernels raise an
  overflow flag instead and the call replays with grown capacities.  A test
  hook starts the call from tiny capacities, and the replayed table must
  equal the oracle's.
"""
import ctypes
import threading
import time

import numpy as np
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200 import _ffi
from gpu_tracking_b200._params import COLUMN_INDEX, trackpy_params
from synth import video

pytestmark = pytest.mark.gpu


def _long_host_video():
    """2048 frames of 1024x1024 uint16 in pageable host memory (4 GiB): the
    call copies them in 128-frame super-chunks, each a blocking host copy, so
    it runs for a good fraction of a second."""
    torch = pytest.importorskip("torch")
    from gpu_tracking_b200.synth import brownian_video
    base = brownian_video(16, 1024, 1024, 400, seed=5, device="cuda").cpu().numpy()
    del torch
    return np.ascontiguousarray(np.tile(base, (128, 1, 1)))


def _watch_and_interrupt(ctx, samples, stop, trigger_done):
    while not stop.is_set():
        d, t = ctx.progress()
        samples.append((d, t))
        if t > 0 and d >= trigger_done:
            ctx.interrupt(True)
            return
        time.sleep(0.0005)


def test_interrupt_mid_call_through_the_c_abi():
    frames = _long_host_video()
    T, H, W = frames.shape
    ctx = _ffi.context(0)
    p = trackpy_params(9, minmass=300.0, search_range=5.0, memory=1)
    out = ctypes.c_void_p()
    samples, stop = [], threading.Event()
    ctx.interrupt(False)
    watcher = threading.Thread(target=_watch_and_interrupt, args=(ctx, samples, stop, 256))
    watcher.start()
    try:
        st = _ffi.lib().gt_batch(ctx.handle, ctypes.byref(p), frames.ctypes.data_as(ctypes.c_void_p), 0, T, H, W,
                                 None, None, 0, ctypes.byref(out))
    finally:
        stop.set()
        watcher.join()
        ctx.interrupt(False)
    assert st == 9, "expected GT_ERR_INTERRUPTED, got %d" % st
    assert not out.value
    done, total = ctx.progress()
    assert total == T and 256 <= done < T
    # the context still works
    small, _ = video(3, 64, 64, 10, seed=1)
    assert len(gt.batch(small, 7, minmass=100.0, tqdm=False)) > 0


def test_interrupt_raises_keyboard_interrupt_and_progress_is_monotone():
    frames = _long_host_video()
    ctx = _ffi.context(0)
    samples, stop = [], threading.Event()
    watcher = threading.Thread(target=_watch_and_interrupt, args=(ctx, samples, stop, 384))
    watcher.start()
    try:
        with pytest.raises(KeyboardInterrupt):
            gt.batch(frames, 9, minmass=300.0, search_range=5.0, tqdm=False)
    finally:
        stop.set()
        watcher.join()
        ctx.interrupt(False)
    # samples of this call (the watcher may first see the previous call's count)
    ds = [d for d, t in samples if t == len(frames)]
    assert ds and all(a <= b for a, b in zip(ds, ds[1:]))


def test_progress_rises_to_the_total():
    frames, _ = video(300, 64, 64, 8, seed=6)
    ctx = _ffi.context(0)
    samples, stop = [], threading.Event()

    def watch():
        while not stop.is_set():
            samples.append(ctx.progress())
            time.sleep(0.0002)

    th = threading.Thread(target=watch)
    th.start()
    try:
        df = gt.batch(frames, 7, minmass=100.0, search_range=4.0, tqdm=False)
    finally:
        stop.set()
        th.join()
    assert len(df) > 0
    done, total = ctx.progress()
    assert (done, total) == (300, 300)
    ds = [d for d, t in samples if t == 300]
    assert all(a <= b for a, b in zip(ds, ds[1:]))
    assert all(0 <= d <= 300 for d in ds)


def _set_caps(ctx, cand, feat):
    L = _ffi.lib()
    L.gt__set_capacities.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]
    L.gt__set_capacities.restype = ctypes.c_int32
    L.gt__get_capacities.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    L.gt__get_capacities.restype = ctypes.c_int32
    old_c, old_f = ctypes.c_int64(), ctypes.c_int64()
    ctx.check(L.gt__get_capacities(ctx.handle, ctypes.byref(old_c), ctypes.byref(old_f)))
    ctx.check(L.gt__set_capacities(ctx.handle, cand, feat))
    return old_c.value, old_f.value


@pytest.mark.parametrize("cand,feat", [(16, 0), (0, 8), (4, 2)])
def test_capacity_overflow_replays_to_the_oracle_table(oracle, cand, feat):
    frames, _ = video(6, 160, 192, 60, seed=7, D=0.8)
    kw = dict(minmass=200.0, search_range=5.0, memory=2)
    tab = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    ctx = _ffi.context(0)
    old = _set_caps(ctx, cand, feat)
    try:
        df = gt.batch(frames, 9, tqdm=False, **kw)
        now = ctypes.c_int64(), ctypes.c_int64()
        _ffi.lib().gt__get_capacities(ctx.handle, ctypes.byref(now[0]), ctypes.byref(now[1]))
        # the capacities grew from the tiny start
        if cand:
            assert now[0].value > cand
        if feat:
            assert now[1].value > feat
    finally:
        _set_caps(ctx, max(old[0], 1), max(old[1], 1))
    assert len(df) == len(tab) and len(df) > 0
    for name in ("frame", "particle", "duration"):
        assert np.array_equal(df[name].to_numpy().astype(np.int64), tab[:, COLUMN_INDEX[name]].astype(np.int64))
    for name in ("y", "x", "mass", "Rg", "ecc", "raw_mass_corrected"):
        a = df[name].to_numpy().astype(np.float32)
        b = tab[:, COLUMN_INDEX[name]].astype(np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
