"""Primaries across GPUs: one process per GPU, each transporting a contiguous
range of the primaries (or of the events) on its own device.

Every primary keeps the MRG32k3a substream of its global index
(first_substream + index), so the tracks, and the summed tallies, do not
depend on how many GPUs share the work.  The only exchange is the final sum of
the FP64 energy-deposit tallies and the counters: one all_reduce through
torch.distributed (NCCL between GPUs, gloo on CPU).  There is no exchange of
tracks during transport: showers are independent.
"""
import numpy as np

# counters that add across ranks; the others are maxima or per-rank timings
SUM_KEYS = ("steps", "substeps", "tracks", "sec_gamma", "sec_electron", "sec_positron", "n_pair", "n_annih",
            "errors", "escaped", "nprim")
MAX_KEYS = ("iterations", "peak_in_flight", "kernel_ms")


def partition(n, rank, world):
    """Contiguous [start, stop) of n items for rank (the first n % world ranks
    take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def partition_events(events, nevents, rank, world):
    """Contiguous primary range holding whole events: rank takes events
    [e0, e1) of an even split of the event indices.  `events` must be sorted
    (primaries of an event are consecutive)."""
    ev = np.asarray(events)
    if ev.size and np.any(np.diff(ev) < 0):
        raise ValueError("primaries must be grouped by event (sorted event indices)")
    e0, e1 = partition(nevents, rank, world)
    return int(np.searchsorted(ev, e0, "left")), int(np.searchsorted(ev, e1, "left"))


def shard(prims, rank, world, nevents=None):
    """This rank's primaries and the global index of its first one.
    prims = (types, E, pos, dir, events or None); with events, whole events
    go to one rank."""
    types, E, pos, d, ev = prims
    if ev is not None and nevents is not None:
        a, b = partition_events(ev, nevents, rank, world)
    else:
        a, b = partition(len(types), rank, world)
    sub = (types[a:b], E[a:b], pos[a:b], d[a:b], ev[a:b] if ev is not None else None)
    return sub, a


def reduce_results(edep, stats, group=None):
    """Sum a rank's tally tensor (in place) and counters over the group; the
    iteration count, peak population and kernel time are maxima."""
    import torch
    import torch.distributed as dist
    dist.all_reduce(edep, group=group)
    dev = edep.device
    s = torch.tensor([float(stats.get(k, 0)) for k in SUM_KEYS], dtype=torch.float64, device=dev)
    m = torch.tensor([float(stats.get(k, 0)) for k in MAX_KEYS], dtype=torch.float64, device=dev)
    dist.all_reduce(s, group=group)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    out = dict(stats)
    for k, v in zip(SUM_KEYS, s.tolist()):
        out[k] = v if k == "escaped" else int(round(v))
    for k, v in zip(MAX_KEYS, m.tolist()):
        out[k] = v if k == "kernel_ms" else int(round(v))
    return edep, out


def transport_sharded(cfg, prims, nvol, rank, world, run, group=None):
    """Transport this rank's share of `prims` with `run(cfg, sub_prims)` ->
    (edep tensor [nevents, nvol], stats dict), then sum over the group.
    cfg.first_substream is the substream of global primary 0; it is restored
    on return."""
    nevents = cfg.nevents if prims[4] is not None else None
    sub, first = shard(prims, rank, world, nevents)
    base = cfg.first_substream
    cfg.first_substream = base + first
    try:
        edep, st = run(cfg, sub)
    finally:
        cfg.first_substream = base
    st = dict(st)
    st["nprim"] = len(sub[0])
    return reduce_results(edep, st, group)
