"""N > 1 path on CPU: two gloo ranks shard requests/slabs and combine their
counters and times (no GPU, no data exchange on the solve path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from aapm_lowdosectimagerecon_competition_b200 import serve, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    items = list(range(11))
    mine = shard.shard_round_robin(items, rank, world)
    slab = shard.slice_slab(128, rank, world)
    stats = {"served": len(mine), "work": float(sum(mine)), "wall_s": 1.0 + rank}
    tot = shard.reduce_stats(stats, max_keys=("wall_s",), sum_keys=("served", "work"))
    q.put((rank, mine, slab, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, s0, t0), (_, m1, s1, t1) = res
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    assert s0 == (0, 64) and s1 == (64, 128)
    for t in (t0, t1):
        assert t["served"] == 11 and t["work"] == 55.0 and t["wall_s"] == 2.0


def test_slabs_match_reference_start_indices():
    # startIdx_k = ceil((k - 1) / n * SLN) for k = 1..n (AAPM_script/DD2MutiSlices.m:95-101)
    import math
    for SLN, n in [(512, 3), (100, 7), (5, 4)]:
        starts = [shard.slice_slab(SLN, r, n)[0] for r in range(n)]
        assert starts == [math.ceil(k / n * SLN) for k in range(n)]
        assert shard.slice_slab(SLN, n - 1, n)[1] == SLN


def test_tuner_candidates_and_cache(tmp_path):
    # host logic only: the candidate tile shapes and the cache format
    direct = serve.TileTuner(sat="direct")
    assert direct.candidates(16) == [(8, 2), (8, 1), (4, 4), (4, 2), (4, 1), (2, 4), (2, 2), (2, 1),
                                     (1, 4), (1, 2), (1, 1)]
    assert direct.candidates(2) == [(2, 1), (1, 2), (1, 1)]
    assert serve.TileTuner(sat="hilo").candidates(4) == [(4, 0), (2, 0), (1, 0)]
    cache = tmp_path / "tiles.json"
    cache.write_text('{"3": 2, "16": [4, 2]}')  # a width-only record and a width + z-tiles record
    t = serve.TileTuner(cache_path=str(cache), sat="direct")
    assert t.table == {3: [2, 0], 16: [4, 2]}
    lib = serve.load()
    try:
        assert lib.ddfan_tune_get_zl(3) == 2 and lib.ddfan_tune_get_zl(16) == 4
        assert lib.ddfan_tune_get_nz(16) == 2 and lib.ddfan_tune_get_nz(3) == 4
        assert lib.ddfan_tune_set_nz(16, 3) != 0
    finally:
        for zb in (3, 16):
            lib.ddfan_tune_set_zl(zb, 0)
            lib.ddfan_tune_set_nz(zb, 0)


def test_admission_policy():
    gb = 1e9
    # oldest that fits within the look-ahead window
    assert serve.pick_admission([5 * gb, 2 * gb], used=0, budget=4 * gb, backfill=8) == 1
    assert serve.pick_admission([5 * gb, 2 * gb], used=0, budget=10 * gb, backfill=8) == 0
    assert serve.pick_admission([5 * gb, 2 * gb], used=0, budget=4 * gb, backfill=1) is None
    assert serve.pick_admission([], used=0, budget=4 * gb, backfill=4) is None
    assert serve.pick_admission([3 * gb], used=2 * gb, budget=4 * gb, backfill=4) is None


def _gather_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    SLN = 7
    a, b = shard.slice_slab(SLN, rank, world)
    # slab of a (YN=2, XN=3) image whose slice z holds z + 0.5
    slab = (torch.arange(a, b, dtype=torch.float32) + 0.5).expand(2, 3, b - a).contiguous()
    full = shard.gather_slabs(slab, SLN, rank, world)
    q.put((rank, full.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gather_uneven_slabs():
    """A sharded image comes back whole on every rank (slabs of 4 and 3 of 7
    slices, padded for the all_gather and trimmed)."""
    import torch
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = (torch.arange(7, dtype=torch.float32) + 0.5).expand(2, 3, 7).tolist()
    for _, full in res:
        assert full == expect
