"""batch_sharded with two ranks (gloo on 127.0.0.1) sharing one GPU: each
rank tracks its half of the frames (plus a prefix) with the engine, the
chunk boundary is verified and the ids relabelled, and the table gathered on
rank 0 equals batch() on the whole video in every column, particle ids and
durations included.  The ranks' kernels never wait on each other; they meet
only through gloo on the host."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import gpu_tracking_b200 as gt
        from gpu_tracking_b200 import sharding
        from synth import video
        frames, _ = video(16, 96, 128, 30, seed=77, D=1.2, turnover=0.08)
        kw = dict(minmass=300.0, search_range=6.0, memory=2, tqdm=False)
        df = sharding.batch_sharded(frames, 9, **kw)
        if rank == 0:
            whole = gt.batch(frames, 9, **kw)
            same = len(df) == len(whole) and list(df.columns) == list(whole.columns) and all(
                np.array_equal(df[c].to_numpy(), whole[c].to_numpy()) for c in whole.columns)
            q.put((rank, same, len(df)))
        else:
            q.put((rank, df is None, 0))
    finally:
        dist.destroy_process_group()


def test_batch_sharded_equals_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r, (ok, n)) for r, ok, n in (q.get(timeout=300) for _ in range(2)))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res[0][0] and res[0][1] > 20
    assert res[1][0]
