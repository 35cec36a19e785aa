"""Segments across GPUs: one process per GPU, no collective on the data path.

The reference pursues one segment per call, one call after another
(spikesorting_parallel.py:1312-1322).  Segments are independent, so N GPUs
take disjoint shares of them; the only exchanges are host-side: the spike
trains (integers) gathered on rank 0, and the max over ranks of a timing.

    from spikesorting_fullpursuit_b200.parallel import distributed as D
    results = D.sort_segments_distributed(segments, costs)   # rank 0: all results in order

`segments` are (voltage, sort_info, separability_metrics, n_max_shift_inds)
tuples; `costs` (e.g. samples x templates, or the HBM footprint) balance the
shares.  Every rank must call with the same `segments` order and `costs`.
"""
import torch.distributed as dist


def partition_segments(costs, world):
    """Longest-first greedy assignment of segments to `world` ranks.

    Returns one list of segment indices per rank (ascending).  Deterministic:
    segments are taken by decreasing cost (ties: lower index first) and each
    goes to the rank with the least cost so far (ties: lower rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(world), key=lambda r: (load[r], r))
        shares[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shares]


def max_over_ranks(value, device=None, group=None):
    """The largest `value` over all ranks (every rank gets it); `value` itself
    without a process group.  `device` is where the reduction tensor lives
    (a CUDA device for NCCL, the CPU for gloo)."""
    import torch
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(local, n_segments, group=None):
    """`local` maps segment index -> result on each rank; rank 0 returns the
    list of all `n_segments` results in index order, other ranks None."""
    if not (dist.is_available() and dist.is_initialized()):
        return [local[i] for i in range(n_segments)]
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError("segment %d was sorted by two ranks" % k)
            merged[k] = v
    missing = [i for i in range(n_segments) if i not in merged]
    if missing:
        raise RuntimeError("segments without a result: %s" % missing[:10])
    return [merged[i] for i in range(n_segments)]


def sort_segments_distributed(segments, costs=None, runner=None, group=None, **kwargs):
    """Sort this rank's share of `segments` and gather every result on rank 0.

    `runner(voltage, sort_info, separability_metrics, n_max_shift_inds,
    **kwargs)` defaults to `binary_pursuit()` on this process's current CUDA
    device (keyword arguments such as precision pass through).  Returns the
    results in segment order on rank 0 and None on the other ranks."""
    if runner is None:
        from .binary_pursuit_parallel import binary_pursuit

        def runner(v, si, m, nmax, **kw):
            return binary_pursuit(v, v.dtype, si, m, n_max_shift_inds=nmax, **kw)
    if costs is None:
        costs = [int(s[0].shape[1]) * int(getattr(s[2]['templates'], 'shape', (1,))[0]) for s in segments]
    initialized = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if initialized else 1
    rank = dist.get_rank(group) if initialized else 0
    mine = partition_segments(costs, world)[rank]
    local = {i: runner(*segments[i], **kwargs) for i in mine}
    return gather_results(local, len(segments), group)
