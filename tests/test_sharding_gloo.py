"""The multi-rank path on CPU: world size 2 over gloo (127.0.0.1).

Ranks split frames and videos into contiguous shares, take the maximum of
their timings, sum their counts and gather their tables on rank 0 in rank
order; the engine's kernels are not involved (no GPU here), each rank's
"located" table is made on the host.
"""
import os
import socket
import sys

import numpy as np
import pandas as pd
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from gpu_tracking_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        T = 11
        a, b = sharding.shard_range(T, rank, world)
        # a stand-in for this rank's located frames: 3 rows per frame
        rows = [(f, 10.0 * f + k, float(k)) for f in range(a, b) for k in range(3)]
        df = pd.DataFrame(rows, columns=["frame", "y", "x"])
        got = sharding.gather_tables(df)
        mx = sharding.max_over_ranks(1.5 + rank)
        sm = sharding.sum_over_ranks(len(df))
        q.put((rank, (a, b), None if got is None else got.to_numpy(), mx, sm))
    finally:
        dist.destroy_process_group()


def test_shard_range_covers_every_item_once():
    from gpu_tracking_b200.sharding import shard_range
    for n in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(5, 2, 2)


def test_two_ranks_gather_reduce_over_gloo():
    sys.path.insert(0, ROOT)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, share, table, mx, sm = q.get(timeout=120)
        out[rank] = (share, table, mx, sm)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == (0, 6) and out[1][0] == (6, 11)
    assert out[1][1] is None
    want = np.array([(f, 10.0 * f + k, float(k)) for f in range(11) for k in range(3)])
    assert np.array_equal(out[0][1], want)
    assert out[0][2] == out[1][2] == 2.5
    assert out[0][3] == out[1][3] == 33.0
