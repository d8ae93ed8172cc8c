"""Batched and served OS-SART reconstructions on one GPU.

* `TileTuner` -- the autotuner: times the projector kernels for each
  candidate tile shape (z-tile width; in the direct mode also the z-tiles a
  thread walks) on a bucket's shape and records the fastest in the library
  (ddfan_tune_set_zl, ddfan_tune_set_nz) and in a JSON cache.
* `Engine` -- continuous batching: requests of uneven sizes are admitted, in
  arrival order with back-fill, while the HBM budget (exact per-request
  estimates from ddfan_ossart_estimate_bytes) and the slot count allow; every
  admitted solve keeps its sinogram, image and tables on the device and runs
  its iterations as CUDA-graph replays on its own stream, so admitted solves
  overlap on the GPU; a finished solve frees its memory (stream-ordered, no
  device-wide synchronisation) and the queue is re-examined.
* `run_batch` -- a fixed batch of instances through the engine (config 4).
* `run_serving` -- Poisson arrivals for a wall-clock window (config 5).

There is no counterpart in the reference (it runs one reconstruction per
MATLAB call); the per-request computation is OSSART_AAPM's
(AAPM_script/OSSART_AAPM.m:33-118).
"""
import collections
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import configs, dd2
from ._lib import BACK_MODES, SAT_MODES, load
from .device import OSSART, Plan


# ---------------------------------------------------------------- workloads

def phantom_torch(XN, SLN, dx, seed, device, n=10):
    """Seeded ellipsoid phantom (water cylinder 0.02/mm + n ellipsoids,
    mu in [0, 0.04]/mm) built on the device, float32 (YN, XN, SLN)."""
    rng = np.random.default_rng(seed)
    c = (torch.arange(XN, device=device, dtype=torch.float32) - (XN - 1) / 2.0) * dx
    zc = (torch.arange(SLN, device=device, dtype=torch.float32) - (SLN - 1) / 2.0) * dx
    Y, X = torch.meshgrid(c, c, indexing="ij")
    R = 0.43 * XN * dx
    img = torch.where(X ** 2 + Y ** 2 <= R * R, 0.02, 0.0)[:, :, None].repeat(1, 1, SLN)
    H = max(SLN * dx, dx)
    for _ in range(n):
        cx, cy = rng.uniform(-0.6, 0.6, 2) * R
        cz = rng.uniform(-0.5, 0.5) * H
        a, b = rng.uniform(0.04, 0.3, 2) * R
        cc = rng.uniform(0.2, 0.8) * H
        th = rng.uniform(0, math.pi)
        mu = float(rng.uniform(0.0, 0.04))
        xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        q2 = (xr / a) ** 2 + (yr / b) ** 2
        zz = ((zc - cz) / cc) ** 2
        inside = q2[:, :, None] + zz[None, None, :] <= 1.0
        img = torch.where(inside, torch.tensor(mu, device=device), img)
    return img.contiguous()


class Instance:
    """One reconstruction problem: geometry, measured sinogram (pinned host
    memory), initial image and iteration count."""

    def __init__(self, scan, proj_host, mask, iters, tag=None):
        self.scan = scan
        self.proj_host = proj_host
        self.mask = mask
        self.iters = iters
        self.tag = tag

    @property
    def work(self):
        """Interpolated samples of one OS-SART iteration (S N + V P)."""
        s = self.scan
        return float(s.PN) * s.DNU * s.SLN * s.XN + float(s.XN) * s.YN * s.SLN * s.PN


def make_instance(N, Z, P, seed, device, iters=5, numOfOS=24, I0=1.5e5):
    """A config-4 style instance: side N, Z slices, P views, 736 channels."""
    s = configs.c2(SLN=Z)
    s.dx = 0.7 * 512 / N
    s.XN = s.YN = N
    s.PN = P
    s.numOfOS = min(numOfOS, P)
    s.I0 = I0
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = phantom_torch(N, Z, s.dx, seed, device)
    pl = Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, N, N, Z, P, s.dx, sat="hilo",
              device=device.index)
    prj = pl.proj(torch.from_numpy(s.angles()).to(device), xt)
    pl.close()
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    y = -torch.log(torch.clamp(torch.poisson(I0 * torch.exp(-prj.double()), generator=g), min=1.0) / I0)
    host = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
    host.copy_(y.float())
    return Instance(s, host, s.circular_mask(), iters, tag=(N, Z, P, seed))


# ---------------------------------------------------------------- autotuner

class TileTuner:
    """Measures every valid tile shape for a slice count (4-slice blocks) on
    a representative shape and keeps the fastest: the z-tile width (z-lanes
    per channel or voxel group, 1-8 blocks) and, in the direct mode, how many
    z-tiles each thread walks per decoded footprint (1, 2 or 4)."""

    def __init__(self, cache_path=None, sat="hilo", back="adj"):
        self.cache_path = cache_path
        self.sat = sat
        self.back = back
        self.table = {}    # zblocks -> [zl, nz] (nz 0: not tuned)
        self.timings = {}  # zblocks -> {"zl,nz": ms}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                for k, v in json.load(f).items():
                    self.table[int(k)] = [int(v), 0] if isinstance(v, int) else [int(v[0]), int(v[1])]
        self.apply()

    def apply(self):
        lib = load()
        for zb, (zl, nz) in self.table.items():
            lib.ddfan_tune_set_zl(zb, zl)
            lib.ddfan_tune_set_nz(zb, nz)

    def save(self):
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump({str(k): v for k, v in sorted(self.table.items())}, f, indent=1)

    def candidates(self, zb):
        """(zl, nz) pairs worth timing for zb blocks: every width that fits,
        and in the direct mode every z-tiles-per-thread count its tiles allow."""
        out = []
        for zl in (8, 4, 2, 1):
            if zl > zb:
                continue
            nzt = -(-zb // zl)
            nzs = [nz for nz in (4, 2, 1) if nz == 1 or nzt >= nz] if self.sat == "direct" else [0]
            out += [(zl, nz) for nz in nzs]
        return out

    def tune(self, N, Z, P, device, reps=2):
        """Returns the chosen [zl, nz] for Z slices (nz 0 outside the direct
        mode); times forward + backprojection of P views on an N x N x Z image
        per candidate."""
        lib = load()
        zb = (Z + 3) // 4
        if zb in self.table:
            return self.table[zb]
        s = configs.c2(SLN=Z)
        x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
        dx = 0.7 * 512 / N
        angs = torch.from_numpy(s.angles(P)).to(device)
        vol = torch.rand((N, N, Z), device=device) * 0.02
        best, best_ms, timings = None, float("inf"), {}
        for zl, nz in self.candidates(zb):
            lib.ddfan_tune_set_zl(zb, zl)
            lib.ddfan_tune_set_nz(zb, nz)
            pl = Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, N, N, Z, P, dx, sat=self.sat,
                      device=device.index)
            prj = pl.proj(angs, vol)
            out = torch.empty_like(vol)
            pl.back(angs, prj, out=out, mode=self.back)
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                pl.proj(angs, vol, out=prj)
                pl.back(angs, prj, out=out, mode=self.back)
            e1.record()
            torch.cuda.synchronize(device)
            ms = e0.elapsed_time(e1) / reps
            timings["%d,%d" % (zl, nz)] = round(ms, 4)
            pl.close()
            if ms < best_ms:
                best, best_ms = [zl, nz], ms
        lib.ddfan_tune_set_zl(zb, best[0])
        lib.ddfan_tune_set_nz(zb, best[1])
        self.table[zb] = best
        self.timings[zb] = timings
        return best


# ---------------------------------------------------------------- engine

def pick_admission(queue_bytes, used, budget, backfill):
    """Index of the next queued request to admit, or None: the oldest request
    among the first `backfill` whose device bytes fit in the budget."""
    for i, b in enumerate(queue_bytes[:max(1, backfill)]):
        if used + b <= budget:
            return i
    return None


class _Active:
    __slots__ = ("req", "solver", "stream", "done", "out_dev", "out_host", "bytes", "t_admit", "iter_done")


class Engine:
    """Continuous-batching executor of OS-SART solves on one GPU."""

    def __init__(self, device=0, budget_bytes=150e9, max_active=8, sat="hilo", back="adj",
                 use_graph=True, backfill=8):
        self.device = torch.device("cuda", device)
        self.budget = float(budget_bytes)
        self.max_active = int(max_active)
        self.sat, self.back = sat, back
        self.use_graph = use_graph
        self.backfill = backfill  # how far past the queue head admission may look
        self.queue = collections.deque()
        self.active = []
        self.used = 0.0
        self.finished = []
        self.peak_used = 0.0
        self.peak_active = 0
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(self.max_active)]
        self._free_streams = list(self._streams)

    def estimate(self, inst):
        s = inst.scan
        return float(load().ddfan_ossart_estimate_bytes(s.XN, s.YN, s.DNU, s.SLN, s.PN, s.numOfOS,
                                                        SAT_MODES[self.sat]))

    def submit(self, inst, t_arrival=None):
        req = {"inst": inst, "t_arrival": time.perf_counter() if t_arrival is None else t_arrival,
               "bytes": self.estimate(inst)}
        if req["bytes"] > self.budget:
            raise ValueError("request needs %.2f GB, above the %.2f GB budget" % (req["bytes"] / 1e9,
                                                                                 self.budget / 1e9))
        self.queue.append(req)

    def _admit_one(self, req):
        inst, s = req["inst"], req["inst"].scan
        x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
        st = self._free_streams.pop()
        a = _Active()
        a.req, a.stream, a.bytes = req, st, req["bytes"]
        a.t_admit = time.perf_counter()
        a.solver = OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx,
                          mask=inst.mask, numOfOS=s.numOfOS, useFISTA=s.useFISTA, nonneg=s.nonneg,
                          sat=self.sat, back=self.back, device=self.device.index)
        with torch.cuda.stream(st):
            # pinned host sinogram -> solver memory, asynchronous on the slot's stream
            a.solver.set_sinogram(inst.proj_host, stream=st)
            a.solver.set_image(torch.zeros((s.YN, s.XN, s.SLN), device=self.device), stream=st)
            # one graph replay per iteration, each followed by an event, so the
            # progress of a solve in flight can be read without waiting for it
            a.iter_done = []
            for _ in range(inst.iters):
                a.solver.iterate(1, use_graph=self.use_graph, stream=st)
                ev = torch.cuda.Event()
                ev.record(st)
                a.iter_done.append(ev)
            a.out_dev = a.solver.image(stream=st)
            a.out_host = torch.empty(a.out_dev.shape, dtype=torch.float32, pin_memory=True)
            a.out_host.copy_(a.out_dev, non_blocking=True)
            a.done = torch.cuda.Event()
            a.done.record(st)
        self.used += a.bytes
        self.active.append(a)
        self.peak_used = max(self.peak_used, self.used)
        self.peak_active = max(self.peak_active, len(self.active))

    def _admit(self):
        while self._free_streams and self.queue:
            i = pick_admission([r["bytes"] for r in self.queue], self.used, self.budget, self.backfill)
            if i is None:
                return
            req = self.queue[i]
            del self.queue[i]
            self._admit_one(req)

    def _poll(self):
        still = []
        for a in self.active:
            if a.done.query():
                t = time.perf_counter()
                a.solver.close()
                self.used -= a.bytes
                self._free_streams.append(a.stream)
                r = a.req
                self.finished.append({"tag": r["inst"].tag, "t_arrival": r["t_arrival"],
                                      "t_admit": a.t_admit, "t_done": t, "image": a.out_host,
                                      "iters": r["inst"].iters, "work": r["inst"].work,
                                      "bytes": a.bytes})
            else:
                still.append(a)
        self.active = still

    def step(self):
        self._poll()
        self._admit()

    def progress(self):
        """(iterations, samples) completed so far by the solves still in flight."""
        it = work = 0
        for a in self.active:
            n = sum(1 for ev in a.iter_done if ev.query())
            it += n
            work += n * a.req["inst"].work
        return it, work

    def drain(self, poll_s=0.0005):
        while self.queue or self.active:
            self.step()
            if self.active:
                time.sleep(poll_s)


def latency_stats(finished, t0=None):
    """Latency percentiles of finished requests: arrival to result (p50/p99),
    and its two parts -- queueing (arrival to admission) and service
    (admission to result, the reconstruction itself on a shared GPU)."""
    lat = np.array([f["t_done"] - f["t_arrival"] for f in finished]) if finished else np.zeros(0)
    qd = np.array([f["t_admit"] - f["t_arrival"] for f in finished]) if finished else np.zeros(0)
    sv = np.array([f["t_done"] - f["t_admit"] for f in finished]) if finished else np.zeros(0)
    pct = lambda a, q: float(np.percentile(a, q)) if a.size else None
    return {"p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "mean_s": float(lat.mean()) if lat.size else None,
            "queue_p50_s": pct(qd, 50), "queue_p99_s": pct(qd, 99),
            "service_p50_s": pct(sv, 50), "service_p99_s": pct(sv, 99), "completed": int(lat.size)}


def run_batch(instances, engine):
    """All instances submitted at once; returns wall time, per-instance latencies
    and the aggregate OS-SART iteration and sample rates."""
    torch.cuda.synchronize(engine.device)
    t0 = time.perf_counter()
    for inst in instances:
        engine.submit(inst, t_arrival=t0)
    engine.drain()
    torch.cuda.synchronize(engine.device)
    wall = time.perf_counter() - t0
    fin = engine.finished
    iters = sum(f["iters"] for f in fin)
    work = sum(f["iters"] * f["work"] for f in fin)
    out = {"instances": len(fin), "wall_s": wall, "iters_per_s": iters / wall,
           "samples_per_s": work / wall, "peak_active": engine.peak_active,
           "peak_gb": engine.peak_used / 1e9}
    out.update(latency_stats(fin))
    return out


def run_batched(instances, device=0, sat="direct", back="adj"):
    """All instances as one batch (device.OSSARTBatch): every solver is set up
    and given its sinogram, then each batched iteration advances all of them
    with one launch per kernel kind, subset step and tile class (one CUDA
    graph); instances with fewer iterations are run in a second batch of the
    rest.  Returns wall time (set-up, iterations and result copies included)
    and the aggregate OS-SART iteration and sample rates."""
    from .device import OSSARTBatch
    dev = torch.device("cuda", device)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    solvers = []
    for inst in instances:
        s = inst.scan
        x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
        sv = OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, mask=inst.mask,
                    numOfOS=s.numOfOS, useFISTA=s.useFISTA, nonneg=s.nonneg, sat=sat, back=back,
                    device=dev.index)
        sv.set_sinogram(inst.proj_host)
        sv.set_image(torch.zeros((s.YN, s.XN, s.SLN), device=dev))
        solvers.append(sv)
    t_setup = time.perf_counter() - t0
    done = 0
    remaining = list(range(len(instances)))
    launches = 0
    while remaining:
        n = min(instances[i].iters for i in remaining) - done
        b = OSSARTBatch([solvers[i] for i in remaining])
        launches = max(launches, b.launches_per_iter)
        b.iterate(n)
        b.close()
        done += n
        remaining = [i for i in remaining if instances[i].iters > done]
    images = [sv.image_host() for sv in solvers]
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    for sv in solvers:
        sv.close()
    iters = sum(inst.iters for inst in instances)
    work = sum(inst.iters * inst.work for inst in instances)
    return {"instances": len(instances), "wall_s": wall, "setup_s": t_setup, "iters_per_s": iters / wall,
            "samples_per_s": work / wall, "launches_per_batched_iter": launches, "images": images}


def plain_mex_seconds_per_iter(s, y_host, mask):
    """Seconds of one OS-SART iteration executed the way
    AAPM_script/OSSART_AAPM.m:79-97 drives the mex functions: per subset a
    host-pointer projection call (host -> device image, FP32 prefix sums,
    device -> host sinogram), the residual on the host, a host-pointer
    reference backprojection call, the update on the host; no graphs.  The
    row/column sums (:59-66) are computed first and not timed."""
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    yh = np.asarray(y_host, np.float32)
    hangs = s.hangs()
    x = np.zeros((s.YN, s.XN, s.SLN), np.float32)
    ones_i = np.ones((s.YN, s.XN, 1), np.float32)
    subs = [np.arange(k, s.PN, s.numOfOS) for k in range(s.numOfOS)]
    rows, cols = [], []
    for v in subs:
        h1 = np.ascontiguousarray(hangs[v][:, :1])
        rows.append(dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h1, len(v), s.XN, s.YN, 1,
                                           ones_i, s.dx, mask, sat="fp32"))
        cols.append(dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h1, len(v),
                                           s.XN, s.YN, 1, np.ones((len(v), s.DNU, 1), np.float32), s.dx,
                                           mask, sat="fp32", back="ref"))
    t0 = time.perf_counter()
    for k, v in enumerate(subs):
        h = np.ascontiguousarray(hangs[v])
        prj = dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h, len(v), s.XN, s.YN, s.SLN, x,
                                     s.dx, mask, sat="fp32")
        rs = rows[k]
        nz = np.broadcast_to(rs != 0, prj.shape)
        prj = np.where(nz, (yh[v] - prj) / np.where(rs != 0, rs, 1), prj).astype(np.float32)
        tp = dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, len(v), s.XN, s.YN,
                                    s.SLN, prj, s.dx, mask, sat="fp32", back="ref")
        cs = cols[k]
        tp = np.where(np.broadcast_to(cs != 0, tp.shape), tp / np.where(cs != 0, cs, 1), tp)
        x = np.maximum(x + tp, 0).astype(np.float32)
    return time.perf_counter() - t0


def run_serving(pool, engine, rate_hz=20.0, window_s=20.0, seed=5):
    """Poisson arrivals at rate_hz drawn round-robin from `pool` (instances of
    the config-4 size distribution) for window_s seconds of wall clock.
    Reports offered vs served rates and latency percentiles of the requests
    completed inside the window."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=int(rate_hz * window_s * 3) + 10)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < window_s]
    order = rng.integers(0, len(pool), size=arrivals.size)
    torch.cuda.synchronize(engine.device)
    t0 = time.perf_counter()
    k = 0
    while True:
        now = time.perf_counter() - t0
        while k < arrivals.size and arrivals[k] <= now:
            engine.submit(pool[order[k]], t_arrival=t0 + arrivals[k])
            k += 1
        engine.step()
        if now >= window_s:
            break
        time.sleep(0.0005)
    # iterations finished inside the window: whole solves plus the finished
    # iterations of the solves still in flight
    part_iters, part_work = engine.progress()
    done_in_window = [f for f in engine.finished if f["t_done"] - t0 <= window_s]
    iters = sum(f["iters"] for f in done_in_window) + part_iters
    work = sum(f["iters"] * f["work"] for f in done_in_window) + part_work
    res = {"offered_rate_hz": arrivals.size / window_s, "served_rate_hz": len(done_in_window) / window_s,
           "arrived": int(arrivals.size), "served": len(done_in_window), "queued_at_end": len(engine.queue),
           "active_at_end": len(engine.active), "iters_per_s": iters / window_s,
           "samples_per_s": work / window_s, "in_flight_iters_counted": part_iters,
           "peak_active": engine.peak_active, "peak_gb": engine.peak_used / 1e9, "window_s": window_s}
    res.update(latency_stats(done_in_window))
    # requests still queued are dropped; the ones on the GPU finish before returning,
    # so nothing of the window overlaps whatever runs next
    engine.queue.clear()
    engine.drain()
    return res
