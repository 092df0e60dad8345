"""One process per GPU: sharding of frames and videos and the host-side
collectives around it (torch.distributed; NCCL on GPUs, gloo on CPU).

Locating is independent per frame and per video, so ranks split the work with
no exchange on the data path.  Linking is a time scan per video; a long
video is linked in time chunks, one per rank (``batch_sharded``):

* rank r tracks its frames [a_r, b_r) preceded by a prefix of P frames
  (P = memory + 1 to start with), locating and linking them on its own GPU;
* the linker's state at a_r (src/linking.rs:349-520: the previous frame's
  points with their ids and the memory ring of unused sources, FIFO of
  `memory` frames) is derived from the ids of the last memory + 1 frames,
  once from rank r's run and once from rank r-1's; the two states are
  equivalent when they hold the same detections in the same order and their
  ids correspond one to one.  From an equivalent state the linker takes the
  same decisions (ids are only compared for identity), so rank r's ids from
  a_r on are the true ids up to that correspondence, and ids created after
  a_r are the true ones shifted by the ids all earlier chunks created (a
  prefix sum of per-chunk counts);
* a boundary whose states differ (a memory entry from before the prefix
  changed a subnet) is re-run with a four times longer prefix, down to
  frame 0 if need be, so the result is always exact;
* durations follow from the global ids with the reference's
  DurationBookkeep rules (src/linking.rs:473-520, src/execute_gpu.rs:1164-1181).

The boundary exchange is a few hundred kilobytes (ids of memory + 1
frames); rank 0 gathers the table's columns as arrays.  Not part of the
reference's API (it runs on one device).
"""
__all__ = ["shard_range", "max_over_ranks", "sum_over_ranks", "gather_tables", "gather_columns", "batch_sharded",
           "linker_state", "match_states", "durations_from_ids"]


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


def gather_columns(arr, dst=0):
    """Concatenate every rank's (n_r, k) float64 array on rank `dst` in rank
    order, through tensors (None on the other ranks)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(), dist.get_rank()
    dev = _device()
    arr = np.ascontiguousarray(arr, np.float64)
    k = arr.shape[1]
    n = torch.tensor([arr.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(x.item()) for x in sizes]
    cap = max(max(sizes), 1)
    buf = torch.zeros((cap, k), dtype=torch.float64, device=dev)
    if arr.shape[0]:
        buf[:arr.shape[0]] = torch.from_numpy(arr).to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst)
    if rank != dst:
        return None
    return np.concatenate([parts[r][:sizes[r]].cpu().numpy() for r in range(world)], axis=0)


def _frame_ids(frame_col, ids):
    """{frame: ids of its rows in table order}."""
    out = {}
    for f, i in zip(frame_col.tolist(), ids.tolist()):
        out.setdefault(int(f), []).append(int(i))
    return out


def linker_state(frame_ids, a, memory):
    """The Linker's state before frame a (src/linking.rs:435-520): the
    previous frame's ids, and the memory ring: for each of the frames
    t = a - memory .. a - 1 (oldest first), the detections of frame t - 1
    whose id frame t does not continue, as (frame, row in frame, id)."""
    prev = list(frame_ids.get(a - 1, []))
    ring = []
    for t in range(a - memory, a):
        before = frame_ids.get(t - 1, [])
        now = set(frame_ids.get(t, []))
        ring.append([(t - 1, k, s) for k, s in enumerate(before) if s not in now])
    return prev, ring


def match_states(mine, theirs):
    """The id correspondence {my id: their id} under which two linker states
    are the same state, or None when they differ."""
    prev_a, ring_a = mine
    prev_b, ring_b = theirs
    if len(prev_a) != len(prev_b) or len(ring_a) != len(ring_b):
        return None
    fwd, back = {}, {}

    def pair(x, y):
        if fwd.setdefault(x, y) != y or back.setdefault(y, x) != x:
            return False
        return True

    for x, y in zip(prev_a, prev_b):
        if not pair(x, y):
            return None
    for la, lb in zip(ring_a, ring_b):
        if len(la) != len(lb):
            return None
        for (fa, ka, x), (fb, kb, y) in zip(la, lb):
            if (fa, ka) != (fb, kb) or not pair(x, y):
                return None
    return fwd


def durations_from_ids(frame_col, ids, n_frames, memory):
    """Per-row durations of linked ids, frame by frame as the reference's
    Linker keeps them (DurationBookkeep, src/linking.rs:473-520): an id
    starts at the frame that creates it; when a memory slot leaves the ring
    every id in it gets (frame - start) - memory, and Linker::finish gives
    the ring's ids (frames - start) - (memory - slot) and the last frame's
    ids frames - start.  The duration column reads the entry of the row's
    particle id as stored in float32 (src/execute_gpu.rs:1164-1181)."""
    import collections

    import numpy as np
    frame_col = np.asarray(frame_col, np.int64)
    ids = np.asarray(ids, np.int64)
    n_ids = int(ids.max()) + 1 if len(ids) else 0
    start = np.full(n_ids, -1, np.int64)
    dur = np.zeros(n_ids, np.int64)
    order = np.argsort(frame_col, kind="stable")
    bounds = np.searchsorted(frame_col[order], np.arange(n_frames + 1))
    ring = collections.deque([np.zeros(0, np.int64) for _ in range(memory)])
    prev = np.zeros(0, np.int64)
    for t in range(n_frames):
        cur = ids[order[bounds[t]:bounds[t + 1]]]
        fresh = cur[start[cur] < 0]
        start[fresh] = t
        unused = prev[~np.isin(prev, cur)]
        if memory > 0:
            ring.append(unused)
            leaving = ring.popleft()
            dur[leaving] = (t - start[leaving]) - memory
        else:
            dur[unused] = t - start[unused]
        prev = cur
    for i, slot in enumerate(ring):
        dur[slot] = (n_frames - start[slot]) - (memory - i)
    dur[prev] = n_frames - start[prev]
    as_f32 = ids.astype(np.float32).astype(np.int64)
    if len(as_f32) and (as_f32.max() >= n_ids or as_f32.min() < 0):
        raise ValueError("a particle id stored as float32 has no duration entry (the reference panics here)")
    return dur[as_f32]


def batch_sharded(video, diameter, prefix=None, tracker=None, **kwargs):
    """``batch`` over a (T, Y, X) video with its frames split across the
    ranks of the default process group.  Every rank holds the video (or at
    least its own frames and the ones before them that the prefix needs) and
    tracks its contiguous share; frame numbers stay global.  With
    ``search_range`` the chunks are linked as one video (see the module
    docstring): the table, gathered on rank 0, equals ``batch(video)`` in
    every column, particle ids and durations included.  Returns the table on
    rank 0 and None elsewhere.

    ``prefix`` sets the first prefix length (default memory + 1 frames);
    ``tracker(frames, frame_numbers, search_range, memory, **kwargs)`` replaces
    the per-rank call to ``batch`` (it returns that call's DataFrame)."""
    import numpy as np
    import pandas as pd
    import torch.distributed as dist
    from . import api
    world, rank = dist.get_world_size(), dist.get_rank()
    T = len(video)
    a, b = shard_range(T, rank, world)
    search_range = kwargs.pop("search_range", None)
    memory = int(kwargs.pop("memory", None) or 0)
    kwargs.pop("frames", None)
    if kwargs.get("linker_reset_points") is not None:
        raise ValueError("batch_sharded does not take linker_reset_points")
    kwargs.setdefault("tqdm", False)

    def track(f0, f1, linked):
        if f1 <= f0:
            return None
        if tracker is not None:
            return tracker(video[f0:f1], range(f0, f1), search_range if linked else None, memory, **kwargs)
        extra = dict(search_range=search_range, memory=memory) if linked else {}
        # frames= selects frames f0 .. f1-1 of the video and keeps their
        # global numbers in the table
        return api.batch(video, diameter, frames=range(f0, f1), **kwargs, **extra)

    if search_range is None:
        part = track(a, b, False)
        cols = list(part.columns) if part is not None and len(part) else None
        names = [c for c in dist_all_gather_object(cols) if c is not None]
        cols = names[0] if names else None
        arr = part[cols].to_numpy(np.float64) if cols and part is not None and len(part) else \
            np.zeros((0, len(cols) if cols else 1))
        full = gather_columns(arr)
        if rank != 0 or not cols:
            return None
        return _frame_from(full, cols)

    P = memory + 1 if prefix is None else max(1, int(prefix))
    p0 = max(0, a - P)
    run = track(p0, b, True)
    while True:
        fr = run["frame"].to_numpy(np.int64) if run is not None else np.zeros(0, np.int64)
        ids = run["particle"].to_numpy(np.int64) if run is not None else np.zeros(0, np.int64)
        fids = _frame_ids(fr, ids)
        # a run from frame 0 is the true run; otherwise its state at a must
        # equal the one the previous rank's run hands over at the same frame
        true_run = p0 == 0
        tail_known = true_run or b - memory - 1 >= p0
        tails = dist_all_gather_object(linker_state(fids, b, memory) if tail_known else None)
        psi = None
        ok = True
        if not true_run:
            theirs = tails[rank - 1]
            psi = match_states(linker_state(fids, a, memory), theirs) if theirs is not None else None
            ok = psi is not None
        if all(dist_all_gather_object(ok)):
            break
        if not ok:
            P *= 4
            p0 = max(0, a - P)
            run = track(p0, b, True)
    # ids are created in increasing order: those below c_r exist before a
    before = ids[fr < a]
    c_r = int(before.max()) + 1 if len(before) else 0
    n_new = max(0, (int(ids.max()) + 1 - c_r) if len(ids) else 0)
    info = dist_all_gather_object((c_r, n_new, psi, true_run, a - p0))
    C = [0] * world
    for r in range(1, world):
        C[r] = C[r - 1] + info[r - 1][1]

    def global_id(r, s):
        while True:
            c, _, m, is_true, _ = info[r]
            if is_true:
                return s
            if s >= c:
                return C[r] + (s - c)
            if s not in m:
                raise RuntimeError("chunk linking: id %d of rank %d is not in its boundary state" % (s, r))
            s = m[s]
            r -= 1

    mine = fr >= a
    chunk = run[mine].reset_index(drop=True) if run is not None else None
    if chunk is not None and len(chunk):
        g = np.fromiter((global_id(rank, int(x)) for x in ids[mine]), np.int64, count=int(mine.sum()))
        # the particle column holds ids as the reference stores them (float32)
        chunk["particle"] = g.astype(np.float32).astype(np.int64)
        chunk["_gid"] = g
    cols = list(chunk.columns) if chunk is not None and len(chunk) else None
    names = [c for c in dist_all_gather_object(cols) if c is not None]
    cols = names[0] if names else None
    arr = chunk[cols].to_numpy(np.float64) if cols and chunk is not None and len(chunk) else \
        np.zeros((0, len(cols) if cols else 1))
    full = gather_columns(arr)
    if rank != 0 or not cols:
        return None
    df = _frame_from(full, cols)
    df["duration"] = durations_from_ids(df["frame"].to_numpy(np.int64), df["_gid"].to_numpy(np.int64), T, memory)
    df = df.drop(columns=["_gid"])
    # the prefix every rank's final run needed (frames before its chunk)
    df.attrs["prefix_frames"] = [x[4] for x in info]
    return df


def dist_all_gather_object(obj):
    """Every rank's small picklable object, in rank order."""
    import torch.distributed as dist
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def _frame_from(full, cols):
    import numpy as np
    import pandas as pd
    df = pd.DataFrame(full, columns=cols)
    for c in ("frame", "particle", "duration", "_gid"):
        if c in df.columns:
            df[c] = df[c].to_numpy(np.float64).astype(np.int64)
    for c in df.columns:
        if c not in ("frame", "particle", "duration", "_gid"):
            df[c] = df[c].astype(np.float64)
    return df
