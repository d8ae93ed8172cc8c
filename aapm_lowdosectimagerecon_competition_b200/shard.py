"""Multi-GPU sharding of reconstructions: one process per GPU, no data exchange.

Slices and requests are independent through the whole OS-SART solve (the
reference splits slices over GPUs the same way, AAPM_script/DD2MutiSlices.m:95-101,
with host-side split/gather), so ranks only agree on who solves what and
combine their timings/counters at the end.
"""
import torch
import torch.distributed as dist


def shard_round_robin(items, rank, world):
    """Items rank, rank + world, ... (requests to this rank)."""
    return list(items)[rank::world]


def slice_slab(SLN, rank, world):
    """[start, stop) slices of this rank's contiguous slab, starts
    ceil(k / world * SLN) like the reference's startIdx."""
    start = -(-rank * SLN // world)
    stop = -(-(rank + 1) * SLN // world)
    return start, stop


def reduce_stats(stats, max_keys=(), sum_keys=(), group=None):
    """All-reduce selected numeric fields across ranks: max for times, sum for
    counts.  Every rank calls it with the same keys (a collective)."""
    if not (dist.is_available() and dist.is_initialized()):
        return dict(stats)
    out = dict(stats)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    for keys, op in ((max_keys, dist.ReduceOp.MAX), (sum_keys, dist.ReduceOp.SUM)):
        if not keys:
            continue
        t = torch.tensor([float(stats[k]) for k in keys], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op, group=group)
        for k, v in zip(keys, t.tolist()):
            out[k] = v
    return out
