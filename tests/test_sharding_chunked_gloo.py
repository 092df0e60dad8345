"""Chunked-time linking across ranks (gpu_tracking_b200/sharding.py), on CPU.

Each rank tracks its contiguous share of a video's frames plus a prefix of
earlier frames; the linker states at every chunk boundary are compared, a
mismatch re-runs that rank with a longer prefix, and ids are relabelled with
a prefix sum of per-chunk new-id counts.  The gathered table must equal one
whole-video run in every column, particle ids and durations included.

The ranks are gloo processes on 127.0.0.1; each rank's tracker is the CPU
oracle (the engine's kernels need a GPU), so these tests check the host-side
protocol: boundary states, the prefix growth, the relabelling and the
durations.  Helpers of the protocol are also checked on their own.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def oracle_tracker(diameter):
    """A per-rank tracker with batch's output columns, made by the oracle."""
    def track(frames, frame_numbers, search_range, memory, **kw):
        import pandas as pd

        from gpu_tracking_b200._params import COLUMN_INDEX, column_names, trackpy_params
        from oracle import loader
        kw = {k: v for k, v in kw.items() if k not in ("tqdm",)}
        if search_range is not None:
            kw.update(search_range=search_range, memory=memory)
        p = trackpy_params(diameter, **kw)
        tab = loader.batch(p, np.asarray(frames, np.float32), frame_numbers=np.asarray(list(frame_numbers)))
        cols = [n for n, _ in column_names(p)]
        df = pd.DataFrame({c: tab[:, COLUMN_INDEX[c]] for c in cols})
        for c in ("frame", "particle", "duration"):
            if c in df:
                df[c] = df[c].astype(np.int64)
        return df
    return track


def worker(rank, world, port, q, case):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    import datetime

    import torch.distributed as dist
    from gpu_tracking_b200 import sharding
    from synth import video
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        T, n, kw, prefix = case
        frames, _ = video(T, 64, 72, n, seed=31 + T, D=1.5, turnover=0.1)
        df = sharding.batch_sharded(frames, 9, prefix=prefix, tracker=oracle_tracker(9), **kw)
        q.put((rank, None if df is None else (list(df.columns), df.to_numpy(np.float64),
                                              df.attrs.get("prefix_frames"))))
    finally:
        dist.destroy_process_group()


def run_ranks(world, case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q, case)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, res = q.get(timeout=300)
        out[rank] = res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


CASES = [
    (2, (14, 14, dict(minmass=200.0, search_range=6.0, memory=0), None)),
    (2, (16, 14, dict(minmass=200.0, search_range=6.0, memory=3), None)),
    (3, (21, 16, dict(minmass=200.0, search_range=7.0, memory=2), None)),
    # a one-frame prefix cannot carry a memory of 3: the boundaries fail and
    # are re-run with longer prefixes
    (3, (24, 16, dict(minmass=200.0, search_range=7.0, memory=3), 1)),
    (2, (10, 12, dict(minmass=200.0), None)),   # no linking: located rows only
]


@pytest.mark.parametrize("world,case", CASES)
def test_chunked_linking_equals_one_run(oracle, world, case):
    sys.path.insert(0, HERE)
    from gpu_tracking_b200._params import COLUMN_INDEX, trackpy_params
    from synth import video
    out = run_ranks(world, case)
    assert all(out[r] is None for r in range(1, world))
    cols, got, prefixes = out[0]
    T, n, kw, prefix = case
    if prefix == 1:
        # some boundary could not be verified from one frame and was re-run
        assert max(prefixes) > 1, prefixes
    frames, _ = video(T, 64, 72, n, seed=31 + T, D=1.5, turnover=0.1)
    want = oracle.batch(trackpy_params(9, **kw), frames.astype(np.float32))
    assert got.shape[0] == len(want) > 0
    for j, c in enumerate(cols):
        w = want[:, COLUMN_INDEX[c]]
        if c in ("frame", "particle", "duration"):
            assert np.array_equal(got[:, j].astype(np.int64), w.astype(np.int64)), c
        else:
            assert np.array_equal(got[:, j].astype(np.float32).view(np.uint32), w.astype(np.float32).view(np.uint32)), c


def test_durations_from_ids_match_the_linker(oracle):
    from gpu_tracking_b200._params import COLUMN_INDEX, trackpy_params
    from gpu_tracking_b200.sharding import durations_from_ids
    sys.path.insert(0, HERE)
    from synth import video
    frames, _ = video(12, 64, 72, 14, seed=5, D=1.5, turnover=0.15)
    for memory in (0, 1, 3):
        tab = oracle.batch(trackpy_params(9, minmass=200.0, search_range=6.0, memory=memory), frames.astype(np.float32))
        fr = tab[:, COLUMN_INDEX["frame"]].astype(np.int64)
        ids = tab[:, COLUMN_INDEX["particle"]].astype(np.int64)
        got = durations_from_ids(fr, ids, len(frames), memory)
        assert np.array_equal(got, tab[:, COLUMN_INDEX["duration"]].astype(np.int64)), memory


def test_match_states_requires_a_one_to_one_correspondence():
    from gpu_tracking_b200.sharding import linker_state, match_states
    a = {0: [0, 1, 2], 1: [0, 3, 1]}
    b = {0: [7, 8, 9], 1: [7, 5, 8]}
    assert match_states(linker_state(a, 2, 1), linker_state(b, 2, 1)) == {0: 7, 3: 5, 1: 8, 2: 9}
    c = {0: [7, 8, 9], 1: [7, 7, 8]}        # two rows share an id that are distinct in a
    assert match_states(linker_state(a, 2, 1), linker_state(c, 2, 1)) is None
    d = {0: [7, 8, 9], 1: [7, 5, 9]}        # a different row left the ring
    assert match_states(linker_state(a, 2, 1), linker_state(d, 2, 1)) is None
