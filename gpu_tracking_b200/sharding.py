"""One process per GPU: sharding of frames and videos and the host-side
collectives around it (torch.distributed; NCCL on GPUs, gloo on CPU).

Locating is independent per frame and per video, so ranks split the work with
no exchange on the data path; linking is a time scan per video and runs where
a whole video's detections are.  ``batch_sharded`` locates a long video's
frames across the ranks and links the gathered detections once on rank 0:
the table equals ``batch(video)`` (frames carry their global numbers, and the
linker sees the same rows in the same order).  Not part of the reference's
API (it runs on one device).
"""
__all__ = ["shard_range", "max_over_ranks", "sum_over_ranks", "gather_tables", "batch_sharded"]


def shard_range(n, rank, world):
    """Contiguous [start, end) share of n items for `rank` of `world`; the
    first n % world ranks take one item more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d of world %d" % (rank, world))
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x):
    """Maximum of a number over all ranks (every rank gets it)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    """Sum of a number over all ranks (every rank gets it)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t)
    return float(t.item())


def gather_tables(df, dst=0):
    """Concatenate every rank's DataFrame on rank `dst`, in rank order (None
    on the other ranks)."""
    import pandas as pd
    import torch.distributed as dist
    world, rank = dist.get_world_size(), dist.get_rank()
    parts = [None] * world if rank == dst else None
    dist.gather_object(df, parts, dst=dst)
    if rank != dst:
        return None
    parts = [p for p in parts if p is not None]
    return pd.concat(parts, ignore_index=True) if parts else None


def batch_sharded(video, diameter, **kwargs):
    """``batch`` over a (T, Y, X) video with its frames split across the
    ranks of the default process group: each rank locates its contiguous
    share (frame numbers stay global), rank 0 gathers the detections and, when
    ``search_range`` is given, links them (the particle column; no duration
    column).  Returns the table on rank 0 and None elsewhere."""
    import torch.distributed as dist
    from . import api
    world, rank = dist.get_world_size(), dist.get_rank()
    T = len(video)
    a, b = shard_range(T, rank, world)
    search_range = kwargs.pop("search_range", None)
    memory = kwargs.pop("memory", None)
    kwargs.pop("frames", None)
    # frames= keeps the global frame numbers in the table
    part = api.batch(video, diameter, frames=range(a, b), **kwargs) if b > a else None
    df = gather_tables(part)
    if rank != 0 or df is None:
        return df
    df = df.sort_values("frame", kind="stable").reset_index(drop=True)
    if search_range is not None and len(df):
        df["particle"] = api.link(df[["frame", "y", "x"]].to_numpy(), search_range, memory=memory or 0)
    return df
