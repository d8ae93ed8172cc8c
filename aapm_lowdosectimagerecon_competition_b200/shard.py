"""Multi-GPU sharding of reconstructions: one process per GPU, no data exchange.

Slices and requests are independent through the whole OS-SART solve (the
reference splits slices over GPUs the same way, AAPM_script/DD2MutiSlices.m:95-101,
with host-side split/gather), so ranks only agree on who solves what and
combine their timings/counters, or gather a sharded image, at the end.
"""
import numpy as np
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


def _slice_equal(h, i, j):
    a, b = np.ascontiguousarray(h[:, i]), np.ascontiguousarray(h[:, j])
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _take(x, a, b, lead):
    """Slices [a, b) of x along its last axis (numpy or torch), slice 0 first
    when lead; contiguous."""
    if isinstance(x, torch.Tensor):
        parts = ([x[..., :1]] if lead else []) + [x[..., a:b]]
        return torch.cat(parts, dim=-1).contiguous()
    parts = ([x[..., :1]] if lead else []) + [x[..., a:b]]
    return np.ascontiguousarray(np.concatenate(parts, axis=-1))


def solve_slab(x0, y0, DNU, xds, yds, detCntIdx, hangs, XN, YN, dx, proj, init, numOfIter, rank, world,
               mask=None, numOfOS=1, useFISTA=1, nonneg=0, sat="hilo", back="ref", device=None):
    """OS-SART (AAPM_script/OSSART_AAPM.m) on this rank's slab of one
    reconstruction, for instances larger than one GPU: slices
    slice_slab(SLN, rank, world) of hangs (PN, SLN), proj (PN, DNU, SLN) and
    init (YN, XN, SLN) -- numpy arrays or tensors -- solved on this process's
    GPU with no exchange (slices are independent).  The subset weights come
    from slice 0's angle list (OSSART_AAPM.m:61-64) and the solver takes
    them from its first slice, so when the slab's first list differs from
    slice 0's (per-slice lists) global slice 0 is solved as an extra leading
    slice and dropped.  Returns (a, b, image), image a CUDA tensor
    (YN, XN, b - a)."""
    from .device import OSSART
    h = np.asarray(hangs, dtype=np.float32)
    SLN = h.shape[1]
    a, b = slice_slab(SLN, rank, world)
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    if b <= a:
        return a, b, torch.empty((YN, XN, 0), device=dev)
    lead = 1 if (a > 0 and not _slice_equal(h, a, 0)) else 0
    hs = _take(h, a, b, lead)
    sv = OSSART(x0, y0, DNU, xds, yds, detCntIdx, hs, XN, YN, hs.shape[1], dx, mask=mask, numOfOS=numOfOS,
                useFISTA=useFISTA, nonneg=nonneg, sat=sat, back=back, device=dev.index)
    try:
        sv.set_sinogram(_take(proj, a, b, lead))
        sv.set_image(_take(init, a, b, lead))
        sv.iterate(numOfIter)
        img = sv.image()
        torch.cuda.synchronize(dev)
    finally:
        sv.close()
    return a, b, img[..., lead:].contiguous()


def gather_slabs(slab, SLN, rank, world, group=None):
    """The whole image on every rank from each rank's slab (the solve_slab
    split of SLN slices): slabs padded to the largest, one all_gather, then
    concatenated along the slice axis.  Every rank calls it (a collective);
    with no process group it returns the slab."""
    if not (dist.is_available() and dist.is_initialized()) or world == 1:
        return slab
    sizes = [slice_slab(SLN, r, world) for r in range(world)]
    nmax = max(b - a for a, b in sizes)
    pad = torch.zeros(slab.shape[:-1] + (nmax,), dtype=slab.dtype, device=slab.device)
    pad[..., :slab.shape[-1]] = slab
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[..., :b - a] for p, (a, b) in zip(parts, sizes)], dim=-1)
