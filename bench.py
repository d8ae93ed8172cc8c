"""Benchmark: OS-SART iterations/s on the full-reconstruction workload.

Workload (one GPU, or one independent instance per rank): 512 x 512 x 128
slices at 0.7 mm, 2304 views over 360 deg, 736 arc channels at 1.2858 mm,
sid 595 mm, sdd 1085.6 mm, 24 ordered subsets, FISTA momentum and
non-negativity, the reference's backprojector (the one OSSART_AAPM.m
drives; --back adj selects the exact adjoint), the direct mode (every
prefix-sum difference summed from the values it telescopes to; --sat fp32 /
hilo / fp64 selects prefix-sum tables instead);
the sinogram is the log of seeded Poisson counts at I0 = 1.5e5 photons/ray of
a seeded ellipsoid phantom (synthetic stand-in for the AAPM projections).
A step is one OS-SART iteration (one CUDA graph replay, 24 subsets).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `--impl reference` times the FP64 CPU port of
the reference path (oracle/) on this host's cores on a bounded sample of the
same workload, scaled to the full image.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "OS-SART iters/s (512^2x128, 2304 views, 24 subsets)"
UNIT = "iter/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sat", default="direct", choices=["fp32", "hilo", "fp64", "direct"])
    ap.add_argument("--back", default="ref", choices=["ref", "adj"])
    ap.add_argument("--slices", type=int, default=128)
    ap.add_argument("--subsets", type=int, default=24, help="c3: ordered subsets (the configuration has 24)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-modes", action="store_true",
                    help="skip the other precision / backprojector modes timed beside the headline")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the final-image check against the FP64 oracle (and the CPU baseline it times)")
    ap.add_argument("--kernels", action="store_true",
                    help="time only one subset's projector kernels (small case for ncu captures)")
    ap.add_argument("--config", default="c3", choices=["c2", "c3", "c4", "c5", "rebin"],
                    help="c3: the OS-SART contract line; c4: batched uneven reconstructions; "
                         "c5: Poisson-arrival serving")
    ap.add_argument("--views", default="shared", choices=["shared", "rebinned", "rebinned-irregular"],
                    help="c3: one angle list for all slices, or per-slice lists as rebinning makes them "
                         "(slices 36 raw views apart, or 86.07 apart as an AAPM-length scan gives)")
    ap.add_argument("--rotations", type=int, default=10, help="rebin: rotations of raw views")
    ap.add_argument("--rebin-slices", type=int, default=512, help="rebin: target slices")
    ap.add_argument("--instances", type=int, default=32)
    ap.add_argument("--window", type=float, default=20.0)
    ap.add_argument("--rate", type=float, default=20.0, help="c5: the configuration's arrival rate (reported)")
    ap.add_argument("--load", type=float, default=0.8, help="c5: arrival rate as a fraction of measured capacity")
    ap.add_argument("--min-served", type=int, default=100, help="c5: completions the window must allow for")
    return ap.parse_args()


def _c4_instances(args, dev, iters):
    from aapm_lowdosectimagerecon_competition_b200 import configs, serve
    sizes = configs.c4_instances(args.instances)
    tuner = serve.TileTuner(sat=args.sat, back=args.back)
    for zb in sorted({(Z + 3) // 4 for _, Z, _ in sizes}):
        tuner.tune(N=512, Z=4 * zb, P=96, device=dev, reps=1)
    insts = [serve.make_instance(N, Z, P, seed=100 + i, device=dev, iters=iters)
             for i, (N, Z, P) in enumerate(sizes)]
    return insts, tuner


def run_c4(args):
    """Config 4: 32 seeded instances (side 256-768, 8-96 slices, 720-2304 views,
    736 channels), 5 OS-SART iterations each, hi/lo prefix sums, tile widths
    from the autotuner.  All submitted at once; the engine runs up to 8 solves
    concurrently (each a CUDA-graph replay per iteration on its own stream)
    and is compared with the same instances one at a time."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import serve
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    insts, tuner = _c4_instances(args, dev, iters=5)
    res = {}
    for name, k in (("serial", 1), ("streams", 8)):
        eng = serve.Engine(device=0, max_active=k, sat=args.sat, back=args.back)
        res[name] = serve.run_batch(insts, eng)
    batched = None
    if args.sat == "direct":
        batched = serve.run_batched(insts, device=0, sat=args.sat, back=args.back)
        # each instance's image from the batch against its own solve through the engine
        solo = {}
        eng = serve.Engine(device=0, max_active=1, sat=args.sat, back=args.back)
        serve.run_batch(insts[:4], eng)
        for f in eng.finished:
            solo[f["tag"]] = f["image"].numpy()
        batched["equal_to_solo"] = all(np.array_equal(batched["images"][i], solo[insts[i].tag]) for i in range(4))
        del batched["images"]
    for r in res.values():
        r.pop("images", None)
    best = batched if batched else res["streams"]
    line = {"metric": "c4 batched OS-SART iterations/s (32 uneven instances, 5 iterations each)",
            "value": best["iters_per_s"], "unit": "iter/s", "higher_is_better": True,
            "batched": batched, "streams": res["streams"], "serial": res["serial"],
            "speedup_vs_serial": best["iters_per_s"] / res["serial"]["iters_per_s"],
            "streams_vs_serial": res["streams"]["iters_per_s"] / res["serial"]["iters_per_s"],
            "tile_table": {zb: {"zl": v[0], "nz": v[1]} for zb, v in sorted(tuner.table.items())},
            "tile_timings_ms": tuner.timings, "sat": args.sat, "back": args.back, "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_c5(args):
    """Config 5: Poisson arrivals of config-4-sized requests, 10 OS-SART
    iterations each, 150 GB admission budget.  The engine's capacity is
    measured first (the pool submitted at once); arrivals then run at
    --load times that capacity (the configuration's 20 req/s is far above
    what one GPU serves at these sizes, and latency measured above capacity
    only measures queue growth) for a window long enough for at least
    --min-served completions, or --window seconds if longer.  Latency is
    reported whole and split into queueing and service; throughput is
    compared with serial plain-FP32 solves (mex-style host round trips) and
    with serial device-resident FP32 solves of the same pool."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import serve
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    args.instances = min(args.instances, 8)
    pool, tuner = _c4_instances(args, dev, iters=10)
    cap_eng = serve.Engine(device=0, budget_bytes=150e9, max_active=8, sat=args.sat, back=args.back)
    cap = serve.run_batch(pool + pool, cap_eng)
    capacity = cap["instances"] / cap["wall_s"]
    rate = args.load * capacity
    window = max(args.window, 1.1 * args.min_served / rate)
    eng = serve.Engine(device=0, budget_bytes=150e9, max_active=8, sat=args.sat, back=args.back)
    served = serve.run_serving(pool, eng, rate_hz=rate, window_s=window)
    served["capacity_req_per_s"] = capacity
    served["load"] = args.load
    served["configured_rate_hz"] = args.rate
    # serial plain FP32, mex-style (host round trips per subset), one iteration of
    # two pool requests timed and scaled to the pool's mean work per request
    mex_rate = []
    for inst in pool[:2]:
        sec = serve.plain_mex_seconds_per_iter(inst.scan, inst.proj_host.numpy(), inst.mask)
        mex_rate.append(inst.work / sec)
    mex_samples = float(np.mean(mex_rate))
    # serial device-resident solves with FP32 sums and the reference backprojector, no graphs
    plain = serve.Engine(device=0, max_active=1, sat="fp32", back="ref", use_graph=False)
    pb = serve.run_batch(pool, plain)
    line = {"metric": "c5 served OS-SART requests/s (Poisson arrivals at %.2f of capacity, 10 iterations each)"
                      % args.load,
            "value": served["served_rate_hz"], "unit": "req/s", "higher_is_better": True,
            "serving": served,
            "serial_plain_fp32_mex": {"samples_per_s": mex_samples,
                                      "req_per_s": mex_samples / (10 * np.mean([i.work for i in pool]))},
            "serial_device_fp32_ref": {"req_per_s": pb["instances"] / pb["wall_s"],
                                       "iters_per_s": pb["iters_per_s"], "samples_per_s": pb["samples_per_s"]},
            "throughput_vs_serial_plain_mex": served["samples_per_s"] / mex_samples,
            "throughput_vs_serial_device_fp32": served["samples_per_s"] / pb["samples_per_s"],
            "budget_gb": 150, "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_c2(args):
    """Config 2: the projector and both backprojectors at 512^2 x 64 slices,
    2304 views, 736 channels (one call each over all views), in every
    prefix-sum mode: device time per call (CUDA events), algorithmic HBM
    GB/s (4V + 4S per call) and the relative L2 / max-abs error against the
    FP64 oracle on two of the 64 slices (slices are independent; the oracle
    sees the same float inputs)."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    from oracle import oracle as O
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    s = configs.c2(SLN=64)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    vol_h = configs.phantom(s)
    vol = torch.from_numpy(vol_h).to(dev)
    angs_h = s.angles()
    angs = torch.from_numpy(angs_h).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    prj_in = torch.rand((s.PN, s.DNU, s.SLN), device=dev, generator=g) * 2.0
    pick = [0, 37]
    h2 = np.repeat(angs_h[:, None], len(pick), 1)
    nt = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = {"proj": O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h2, s.PN, s.XN, s.YN, len(pick),
                          np.ascontiguousarray(vol_h[:, :, pick]), s.dx, nthreads=nt)}
    pin = np.ascontiguousarray(prj_in.cpu().numpy()[:, :, pick])
    for mode, m in (("back_adj", O.ADJ), ("back_ref", O.REF)):
        ref[mode] = O.back(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h2, s.PN, s.XN, s.YN, len(pick), pin,
                           s.dx, mode=m, nthreads=nt)
    oracle_s = time.perf_counter() - t0
    V, S = s.XN * s.YN * s.SLN, s.PN * s.DNU * s.SLN
    res = {}
    for sat in ("fp32", "hilo", "fp64", "direct"):
        pl = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx, sat=sat)
        out_p = torch.empty((s.PN, s.DNU, s.SLN), device=dev)
        out_b = torch.empty((s.YN, s.XN, s.SLN), device=dev)
        calls = {"proj": lambda: pl.proj(angs, vol, out=out_p),
                 "back_adj": lambda: pl.back(angs, prj_in, out=out_b, mode="adj"),
                 "back_ref": lambda: pl.back(angs, prj_in, out=out_b, mode="ref")}
        row = {}
        for name, fn in calls.items():
            for _ in range(max(args.warmup, 1)):
                fn()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                fn()
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / args.steps
            got = (out_p if name == "proj" else out_b).cpu().numpy()[:, :, pick].astype(np.float64)
            exp = ref[name]
            d = got - exp
            row[name] = {"ms": ms, "alg_gbs": 4.0 * (V + S) / (ms / 1e3) / 1e9,
                         "rel_l2": float(np.linalg.norm(d.ravel()) / np.linalg.norm(exp.ravel())),
                         "max_abs": float(np.abs(d).max()), "ref_max": float(np.abs(exp).max())}
        pl.close()
        res[sat] = row
    peak, peak_kind = peaks()
    # the headline: the fastest of the modes without cancellation in the
    # prefix-sum differences (plain FP32 is reported beside it)
    best = min(("hilo", "fp64", "direct"), key=lambda k: res[k]["proj"]["ms"])
    line = {"metric": "c2 projector calls (512^2x64, 2304 views, 736 channels): forward ms per call",
            "value": res[best]["proj"]["ms"], "unit": "ms", "higher_is_better": False, "best_mode": best,
            "modes": res, "hbm_peak_gbs": peak, "peak_source": peak_kind,
            "parity": {"slices": pick, "against": "FP64 CPU oracle, same float inputs",
                       "bound_compensated": 2e-6, "oracle_seconds": oracle_s, "oracle_cores": nt},
            "config": {"workload": "c2: 512x512x64 at 0.7 mm, 2304 views, 736 channels at 1.2858 mm, "
                                   "sid 595, sdd 1085.6; seeded ellipsoid phantom; one call over all views",
                       "l2": "inputs larger than L2 (sinogram 434 MB)"},
            "steps": args.steps, "warmup": args.warmup, "data": "synthetic"}
    print(json.dumps(line), flush=True)


REBIN_METRIC = "helical-to-fan rebinned slices/s (736x64 detector, 2304 views/rotation, 512 slices)"
REBIN_UNIT = "slices/s"


def rebin_workload(rotations=10, SLN=512):
    """Siemens-like helical scan: 736 channels x 64 rows, 2304 views per
    rotation, pitch 0.8, `rotations` turns of raw views; slice positions
    linspace(h, deltaZ * TotalView - h, SLN) as AAPM_script/reconscript.m:22."""
    f = np.float32
    p = dict(SD=f(1085.6), SO=f(595.0), BVAngle=f(0.0), DetWidth=736, DetHeight=64, PerDetW=f(1.2858),
             PerDetH=f(1.0947), DefTimes=2304, DetCenterW=f(369.625), SpiralPitchFactor=f(0.8))
    TV = rotations * p["DefTimes"]
    h = p["SpiralPitchFactor"] * p["PerDetH"] * f(p["DetHeight"]) * p["SO"] / p["SD"]
    dZ = h / f(p["DefTimes"])
    z = np.linspace(float(h), float(dZ) * TV - float(h), SLN).astype(np.float32)
    return p, TV, z


def rebin_config(p, TV, z):
    return {"workload": "helical-to-fan rebinning: %d raw views of %dx%d, %d views/rotation, %d slices"
                        % (TV, p["DetWidth"], p["DetHeight"], p["DefTimes"], z.size),
            "raw_views": TV, "DetWidth": p["DetWidth"], "DetHeight": p["DetHeight"],
            "DefTimes": p["DefTimes"], "SLN": int(z.size), "pitch": float(p["SpiralPitchFactor"]),
            "l2": "inputs larger than L2 (raw views %.1f GB)" % (TV * p["DetWidth"] * p["DetHeight"] * 4 / 1e9)}


def rebin_cpu_timing(proj, z, p, slices):
    """Seconds per slice of the reference's own CPU HelicalToFan
    (oracle/_ref/libref_rebin.so, kind "reference") on the first `slices`
    slices, else of the numpy restatement (kind "port")."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libref_rebin.so")
    zz = np.ascontiguousarray(z[:slices])
    if os.path.exists(ref):
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        import make_rebin_fixtures as M
        lib = M.load_reference()
        t0 = time.perf_counter()
        M.run_reference(lib, proj, zz, p["SD"], p["SO"], p["BVAngle"], p["DetWidth"], p["DetHeight"],
                        p["PerDetW"], p["PerDetH"], p["DefTimes"], p["DetCenterW"], p["SpiralPitchFactor"])
        return (time.perf_counter() - t0) / slices, "reference", os.cpu_count() or 1
    from oracle import np_oracle as N
    t0 = time.perf_counter()
    N.helical_to_fan(proj, zz, **p)
    return (time.perf_counter() - t0) / slices, "port", 1


def rebin_last_view(p, z):
    """Largest 1-based raw view the slices at z read (HelicalToFanFunc_mex.cpp:66,73)."""
    f = np.float32
    h = p["SpiralPitchFactor"] * p["PerDetH"] * f(p["DetHeight"]) * p["SO"] / p["SD"]
    dZ = h / f(p["DefTimes"])
    starts = np.floor((np.asarray(z, np.float32) - h * f(0.5)) / dZ).astype(np.int64)
    return int(starts.max()) + p["DefTimes"] - 1


def _rebin_host_raw(p, TV, seed=11):
    rng = np.random.default_rng(seed)
    return rng.random((TV, p["DetWidth"], p["DetHeight"]), dtype=np.float32)


def run_rebin_reference(args):
    """--impl reference --config rebin: the reference's CPU rebinning on a
    bounded sample of slices per step (rank 0 only)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    p, TV, z = rebin_workload(args.rotations, args.rebin_slices)
    sample = min(32, z.size)
    # only the raw views the sampled slices read are generated
    proj = _rebin_host_raw(p, min(TV, rebin_last_view(p, z[:sample])))
    rebin_cpu_timing(proj, z, p, 2)
    per = []
    kind, cores = "reference", 1
    for _ in range(args.steps):
        sec, kind, cores = rebin_cpu_timing(proj, z, p, sample)
        per.append(sec)
    sec = statistics.mean(per)
    v = 1.0 / sec
    line = {"impl": "reference", "metric": REBIN_METRIC, "value": v, "unit": REBIN_UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * z.size * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": rebin_config(p, TV, z),
            "cpu_baseline": {"value": v, "unit": REBIN_UNIT, "cores": cores, "kind": kind,
                             "sample": "first %d of %d slices per step; the reference starts one thread per "
                                       "core but every thread's slice range begins at 0 "
                                       "(HelicalToFanFunc_mex.cpp:165-181), so the last thread rebins all "
                                       "of them" % (sample, z.size)},
            "e2e": {"value": v, "unit": REBIN_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_rebin(args):
    """--config rebin: GPU rebinning of the whole scan per step."""
    import ctypes
    import torch
    import torch.distributed as dist
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    from aapm_lowdosectimagerecon_competition_b200._lib import call

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    p, TV, z = rebin_workload(args.rotations, args.rebin_slices)
    SLN, T, W, H = z.size, p["DefTimes"], p["DetWidth"], p["DetHeight"]
    g = torch.Generator(device=dev)
    g.manual_seed(11 + rank)
    d_raw = torch.rand((TV, W, H), generator=g, device=dev, dtype=torch.float32)
    d_out = torch.empty((T, W, SLN), device=dev, dtype=torch.float32)
    d_views = torch.empty((T, SLN), device=dev, dtype=torch.float32)
    stream = torch.cuda.current_stream(dev)
    zp = z.ctypes.data_as(ctypes.c_void_p)
    V = lambda t: ctypes.c_void_p(t.data_ptr())

    def launch(layout, out=d_out, views=d_views):
        call("ddfan_helical_to_fan_dev", V(d_raw), TV, zp, SLN, p["SD"], p["SO"], p["BVAngle"], W, H,
             p["PerDetW"], p["PerDetH"], T, p["DetCenterW"], p["SpiralPitchFactor"], layout, V(out), V(views),
             ctypes.c_void_p(stream.cuda_stream))

    for _ in range(max(args.warmup, 3)):
        launch(1)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        launch(1)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_per_step = ms_max / args.steps
    value = world * SLN * args.steps / (ms_max / 1e3)

    # mex layout (reference output order), for the roofline comparison
    d_out0 = torch.empty((SLN, T, W), device=dev, dtype=torch.float32)
    d_views0 = torch.empty((SLN, T), device=dev, dtype=torch.float32)
    launch(0, d_out0, d_views0)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e2.record(stream)
    for _ in range(args.steps):
        launch(0, d_out0, d_views0)
    e3.record(stream)
    torch.cuda.synchronize(dev)
    ms_mex = e2.elapsed_time(e3) / args.steps
    same = bool(torch.equal(d_out0.permute(1, 2, 0), d_out) and torch.equal(d_views0.t(), d_views))
    del d_out0, d_views0

    # algorithmic bytes: every raw view some slice reads (all of them here) + the outputs
    f = np.float32
    h = p["SpiralPitchFactor"] * p["PerDetH"] * f(H) * p["SO"] / p["SD"]
    dZ = h / f(T)
    starts = np.floor((z - h * f(0.5)) / dZ).astype(np.int64)
    lo, hi = max(1, int(starts.min())), int(starts.max()) + T - 1
    raw_bytes = (hi - lo + 1) * W * H * 4
    alg = raw_bytes + SLN * T * W * 4 + SLN * T * 4
    peak, peak_kind = peaks()
    achieved = alg / (ms_per_step / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "k_rebin_routine_siemens512.md")) as fh:
            for ln in fh:
                if ln.startswith("traffic_bytes_per_launch:"):
                    traffic = float(ln.split(":", 1)[1])
    except OSError:
        pass
    roofline = {"bound": "hbm", "kernel": "k_rebin_routine", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic, "algorithmic_bytes": alg,
                "launch_ms": ms_per_step, "mex_layout_launch_ms": ms_mex, "layouts_agree": same,
                "note": "algorithmic bytes = raw views read once + rebinned sinogram + view angles"}
    line = {"metric": REBIN_METRIC, "value": value, "unit": REBIN_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": rebin_config(p, TV, z),
            "gpu_launches": args.steps, "clocks": clk, "roofline": roofline}

    if not args.no_e2e or (rank == 0 and world == 1 and not args.no_cpu):
        proj_h = d_raw.cpu().numpy()
    if not args.no_e2e:
        t_e2e = []
        for rep in range(3):
            torch.cuda.synchronize(dev)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            P, Vw = dd2.HelicalToFanFunc_mex(proj_h, z, SLN, **p)
            t_e2e.append(time.perf_counter() - t0)
        te = min(t_e2e[1:] or t_e2e)
        tt = torch.tensor([te], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
        line["e2e"] = {"value": world * SLN / te, "unit": REBIN_UNIT, "h2d_bytes_per_step": int(raw_bytes + SLN * 4),
                       "d2h_bytes_per_step": int(SLN * T * W * 4 + SLN * T * 4),
                       "step": "one ddfan_HelicalToFan call from pageable host arrays (mex layouts): "
                               "upload of the raw views the slices read, rebinning, download",
                       "seconds_per_call": te}
        del P, Vw
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = min(32, SLN)
        sec, kind, cores = rebin_cpu_timing(proj_h, z, p, sample)
        line["cpu_baseline"] = {"value": 1.0 / sec, "unit": REBIN_UNIT, "cores": cores, "kind": kind,
                                "sample": "first %d of %d slices; the reference's thread split gives every "
                                          "thread a range starting at slice 0, so the last thread rebins all"
                                          % (sample, SLN)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_kernels(args):
    """One 96-view subset of the workload through the device Plan API:
    forward, exact-adjoint and reference backprojection, `steps` times each
    after `warmup` rounds.  Prints per-call device ms (CUDA events)."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import dd2, device
    dev = torch.device("cuda", 0)
    s = workload(args.slices, args.subsets)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    angs = torch.from_numpy(np.ascontiguousarray(s.angles()[::s.numOfOS])).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    vol = torch.rand((s.YN, s.XN, s.SLN), device=dev, generator=g) * 0.02
    pl = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, angs.numel(), s.dx,
                     sat=args.sat)
    prj = pl.proj(angs, vol)
    out = torch.empty_like(vol)
    calls = {"proj": lambda: pl.proj(angs, vol, out=prj),
             "back_adj": lambda: pl.back(angs, prj, out=out, mode="adj"),
             "back_ref": lambda: pl.back(angs, prj, out=out, mode="ref")}
    res = {}
    for name, fn in calls.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name + "_ms"] = e0.elapsed_time(e1) / max(args.steps, 1)
    pl.close()
    print(json.dumps({"kernels": res, "sat": args.sat, "views": int(angs.numel()),
                      "image": [s.XN, s.YN, s.SLN]}), flush=True)


def workload(slices, subsets=24):
    from aapm_lowdosectimagerecon_competition_b200 import configs
    s = configs.c3(SLN=slices)
    s.numOfOS = subsets
    return s


def view_angles(s, views):
    if views == "rebinned":
        return s.rebinned_hangs(spacing=36)
    if views == "rebinned-irregular":
        return s.rebinned_hangs(spacing=86.07)
    return s.hangs()


def config_dict(s, args, n):
    return {"workload": "OS-SART c3: %dx%dx%d, %d views, %d channels, %d subsets, FISTA+nonneg" %
                        (s.XN, s.YN, s.SLN, s.PN, s.DNU, s.numOfOS),
            "image": [s.XN, s.YN, s.SLN], "views": s.PN, "channels": s.DNU, "subsets": s.numOfOS,
            "sat": args.sat, "back": args.back, "instances": n,
            "view_angles": {"shared": "one list shared by all slices",
                            "rebinned": "per-slice lists as helical rebinning makes them, slices 36 raw views apart",
                            "rebinned-irregular": "per-slice lists as helical rebinning makes them, slices 86.07 "
                                                  "raw views apart"}[getattr(args, "views", "shared")],
            "l2": "inputs larger than L2 (sinogram 868 MB, image 134 MB%s)" % (
                "" if args.sat == "direct" else ", prefix-sum tables 0.8 GB"),
            "parallelism": "one independent reconstruction per GPU (slices/requests shard with no exchange)"}


# ----------------------------------------------------------------- CPU port

def cpu_port_timing(s, slices, iters=1, nthreads=None, back="ref"):
    """Seconds per OS-SART iteration of the FP64 CPU port on `slices` slices."""
    from oracle import oracle as O
    from oracle import np_oracle as N
    x0, y0, xds, yds = N.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    h = np.repeat(s.angles()[:, None], slices, 1)
    y = np.zeros((s.PN, s.DNU, slices), np.float32)
    init = np.zeros((s.YN, s.XN, slices), np.float32)
    nt = nthreads or (os.cpu_count() or 1)
    _, secs = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0.0, 0.0, h, s.PN, s.XN, s.YN, slices,
                       y, init, s.dx, None, iters, s.numOfOS, s.useFISTA, s.nonneg,
                       back_mode=O.ADJ if back == "adj" else O.REF, nthreads=nt, timing=True)
    return secs / iters, nt


def run_reference(args):
    """--impl reference: the FP64 CPU port of the reference path (no CPU
    implementation of the path exists in the reference itself)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    s = workload(args.slices, args.subsets)
    sample = 2
    from oracle import oracle as O
    O.build()
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_port_timing(s, 1, 1, back=args.back)
    per = []
    nt = 1
    for _ in range(args.steps):
        sec, nt = cpu_port_timing(s, sample, 1, back=args.back)
        per.append(sec * s.SLN / sample)
    t = statistics.mean(per)
    v = 1.0 / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(s, args, 1),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nt, "kind": "port",
                             "sample": "1 OS-SART iteration (24 subsets, 2304 views) on %d of %d "
                                       "slices per step, scaled by %d/%d (slices are independent)"
                                       % (sample, s.SLN, s.SLN, sample)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm

class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in self.f.read().splitlines():
            c = [x.strip() for x in row.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for name, val in zip(names, c[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


# ncu summaries in profiles/ by (direct mode?, backprojector) and kernel slot
PROFILE_OF = {
    (False, "adj"): {"fwd": "k_fwd_c3_subset.md", "back_a": "k_back_adj_c3_subset.md",
                     "back_b": "k_back_adj_c3_subset.md"},
    (False, "ref"): {"fwd": "k_fwd_c3_subset.md"},
    (True, "adj"): {"fwd": "k_fwd_dd_c3_subset.md", "back_a": "k_back_dd_c3_subset.md",
                    "back_b": "k_back_dd_c3_subset.md"},
    (True, "ref"): {"fwd": "k_fwd_dd_c3_subset.md", "back_a": "k_back_ref_dd_c3_subset.md"},
}


def profiled_traffic(kernel, sat="hilo", back="adj"):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    recorded from an ncu capture of this kernel in profiles/, or None."""
    name = PROFILE_OF[(sat == "direct", back)].get(kernel)
    if not name:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def make_problem(s, dev, seed=7):
    """Phantom, noiseless sinogram (our forward), Poisson log sinogram; all on `dev`."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = torch.from_numpy(configs.phantom(s)).to(dev)
    angs = torch.from_numpy(s.angles()).to(dev)
    pl = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx,
                     sat="fp64", device=dev.index)
    prj = pl.proj(angs, xt)
    pl.close()
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    counts = torch.poisson(s.I0 * torch.exp(-prj.double()), generator=g)
    y = (-torch.log(torch.clamp(counts, min=1.0) / s.I0)).float()
    torch.cuda.synchronize(dev)
    return (x0, y0, xds, yds), xt, y


def run_ours(args):
    import torch
    import torch.distributed as dist
    from aapm_lowdosectimagerecon_competition_b200 import dd2, device

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    s = workload(args.slices, args.subsets)
    (x0, y0, xds, yds), xt, y = make_problem(s, dev, seed=7 + rank)
    mask = s.circular_mask()
    hangs = view_angles(s, args.views)
    solver = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, hangs, s.XN, s.YN, s.SLN, s.dx,
                           mask=mask, numOfOS=s.numOfOS, useFISTA=s.useFISTA, nonneg=s.nonneg,
                           sat=args.sat, back=args.back, device=local)
    solver.set_sinogram(y)
    solver.set_image(torch.zeros_like(xt))
    stream = torch.cuda.current_stream(dev)
    solver.iterate(max(args.warmup, 3), use_graph=True, stream=stream)
    torch.cuda.synchronize(dev)

    # ---- timed region: K graph replays, device time on the launching stream
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.iterate(args.steps, use_graph=True, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_per_step = ms_max / args.steps
    value = world * args.steps / (ms_max / 1e3)

    # ---- per-kernel device time (events around every launch, same stream)
    prof = solver.profile(1, stream=stream)
    launches = solver.launches_per_iter * args.steps
    top = max(("fwd", "back_a", "back_b", "sat_image", "sat_sino"), key=lambda k: prof[k][0])
    V = s.XN * s.YN * s.SLN
    S_sub = (s.PN // s.numOfOS) * s.DNU * s.SLN
    # algorithmic bytes per launch (minimum HBM traffic): forward 4V + 4S,
    # backprojection 4S + 4V (read the subset residual table once, write the image)
    alg = {"fwd": 4.0 * (V + S_sub), "back_a": 4.0 * (V + S_sub), "back_b": 4.0 * (V + S_sub),
           "sat_image": 4.0 * V + 2 * 12.0 * V, "sat_sino": 4.0 * S_sub + 12.0 * S_sub}
    if args.sat == "direct":
        # the forward also reads the measured sinogram and writes the residual
        # (the prefix-sum kernels it replaces did that)
        alg["fwd"] = 4.0 * V + 8.0 * S_sub
    top_ms = prof[top][0] / max(prof[top][1], 1)
    peak, peak_kind = peaks()
    achieved = alg[top] / (top_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": profiled_traffic(top, args.sat, args.back), "algorithmic_bytes": alg[top],
                "launch_ms": top_ms,
                "kernel_ms_per_iter": {k: round(v[0], 3) for k, v in prof.items()},
                "note": "achieved = algorithmic bytes per launch / CUDA-event launch time; the "
                        "path is gather/issue bound, not HBM bound"}
    if top == "fwd" and args.views == "shared" and args.sat != "direct":
        # the bound that applies: L1 gathers of prefix-sum cells -- per line of
        # each ray group one cell per boundary (CG channels share CG + 1
        # boundaries), a cell holding 4 slices (32 B FP32, 48 B hi/lo or FP64)
        from aapm_lowdosectimagerecon_competition_b200 import _lib
        cell = {"fp32": 32, "hilo": 48, "fp64": 48}[args.sat]
        zl = int(_lib.load().ddfan_tune_get_zl((s.SLN + 3) // 4))
        cg = 4 if zl >= 4 else (2 if zl == 2 else 1)
        l1_bytes = (s.PN // s.numOfOS) * s.DNU * s.XN * ((s.SLN + 3) // 4) * (1.0 + 1.0 / cg) * cell
        l1_peak = 148 * 128 * 1.965e9 / 1e12  # TB/s: 128 B per clock per SM at the maximum SM clock
        l1_tbs = l1_bytes / (top_ms / 1e3) / 1e12
        roofline["l1_gather"] = {"bytes_per_launch": l1_bytes, "achieved_tbs": l1_tbs, "peak_tbs": l1_peak,
                                 "frac": l1_tbs / l1_peak,
                                 "peak_source": "nominal L1 data bandwidth (148 SMs x 128 B/clk x 1.965 GHz)"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_dict(s, args, world), "gpu_launches": launches,
            "clocks": clk, "roofline": roofline}

    # ---- end to end through the public one-call API with host buffers
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        y_h = pin(y.cpu().numpy())
        x_h = pin(np.zeros((s.YN, s.XN, s.SLN), np.float32))
        out_h = torch.empty((s.YN, s.XN, s.SLN), dtype=torch.float32).pin_memory()
        conf = s.conf()
        e2e_iters = 10
        t_e2e = []
        for rep in range(3):
            torch.cuda.synchronize(dev)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            _ossart_host(s, (x0, y0, xds, yds), y_h, x_h, out_h, mask, e2e_iters, args)
            torch.cuda.synchronize(dev)
            t_e2e.append(time.perf_counter() - t0)
        te = min(t_e2e[1:] or t_e2e)
        tt = torch.tensor([te], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
        h2d = int(y_h.numel() * 4 + x_h.numel() * 4 + s.PN * s.SLN * 4)
        d2h = int(out_h.numel() * 4)
        line["e2e"] = {"value": world * e2e_iters / te, "unit": UNIT,
                       "h2d_bytes_per_step": h2d // e2e_iters, "d2h_bytes_per_step": d2h // e2e_iters,
                       "h2d_bytes_per_call": h2d, "d2h_bytes_per_call": d2h,
                       "step": "one iteration of a ddfan_OSSART_AAPM call (solver set-up, weights, %d "
                               "iterations, pinned H2D of sinogram+image, D2H of the image); bytes per step "
                               "are the call's over its %d iterations" % (e2e_iters, e2e_iters),
                       "seconds_per_call": te}

    # ---- plain FP32 DD, one instance per launch, host round trips per subset
    if not args.no_plain and rank == 0:
        line["plain_fp32"] = plain_fp32_iteration(s, (x0, y0, xds, yds), y, mask)

    # ---- the same iteration in the other modes (compensated tables, the exact adjoint)
    if not args.no_modes and rank == 0:
        modes = {}
        # per-slice lists run on the tables in every mode: only the backprojector varies
        pairs = (("hilo", "ref"), ("hilo", "adj"), ("direct", "adj"), ("direct", "ref")) if args.views == "shared" \
            else ((args.sat, "adj"), (args.sat, "ref"))
        for sat, back in pairs:
            if (sat, back) != (args.sat, args.back):
                modes["%s/%s" % (sat, back)] = mode_rate(s, (x0, y0, xds, yds), y, mask, hangs, sat, back, local)
        line["other_modes"] = {"iters_per_s": modes,
                               "how": "the same workload and sinogram, 2 warm-up and 5 timed graph replays "
                                      "per mode (sat/back); hilo = compensated prefix-sum tables"}

    # ---- final-image parity at this configuration, and the CPU baseline
    parity_failed = False
    if rank == 0 and not args.no_parity:
        par, cpu = parity_check(s, (x0, y0, xds, yds), y, mask, hangs, solver, stream, args)
        line["parity"] = par
        parity_failed = not par["ok"]
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if parity_failed:
        print("PARITY FAILURE: final image rel-L2 %.3g above the bound %.0e against the FP64 oracle"
              % (line["parity"]["rel_l2"], line["parity"]["bound"]), file=sys.stderr, flush=True)
        sys.exit(3)


PARITY_BOUND = 1e-5


def parity_check(s, geom, y, mask, hangs, solver, stream, args):
    """The workload's own final image against the FP64 oracle: the GPU solves
    every slice for s.numOfIter iterations from zero; the oracle solves slices
    0 and 77 of the same sinogram (slices are independent given the subset
    weights, which both take from slice 0's angles, AAPM_script/
    OSSART_AAPM.m:61-64).  The oracle's iteration time is the CPU baseline."""
    import torch
    from oracle import oracle as O
    x0, y0, xds, yds = geom
    iters = s.numOfIter
    solver.set_image(torch.zeros((s.YN, s.XN, s.SLN), device=y.device))
    solver.iterate(iters, use_graph=True, stream=stream)
    torch.cuda.synchronize(y.device)
    xg = solver.image().cpu().numpy().astype(np.float64)
    pick = sorted({0, min(77, s.SLN - 1)})
    ys = np.ascontiguousarray(y.cpu().numpy()[:, :, pick])
    hs = np.ascontiguousarray(np.asarray(hangs)[:, pick])
    init = np.zeros((s.YN, s.XN, len(pick)), np.float32)
    nt = os.cpu_count() or 1
    xo, secs = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0.0, 0.0, hs, s.PN, s.XN, s.YN, len(pick), ys, init,
                        s.dx, mask, iters, s.numOfOS, s.useFISTA, s.nonneg,
                        back_mode=O.ADJ if args.back == "adj" else O.REF, nthreads=nt, timing=True)
    # With per-slice angle lists the reference's update diverges on every slice
    # whose rays differ from slice 0's: the row sums are slice 0's
    # (OSSART_AAPM.m:63), and where a row sum is 0 the residual is replaced by
    # A x itself (:88), so rays that miss slice 0's masked disk but cross this
    # slice's feed the image back into itself.  The bound then applies to
    # slice 0; the other slice is reported (both solves blow up alike).
    bounded = pick if args.views == "shared" else pick[:1]
    sel = [pick.index(z) for z in bounded]
    d = xg[:, :, bounded] - xo[:, :, sel]
    rel = float(np.linalg.norm(d.ravel()) / np.linalg.norm(xo[:, :, sel].ravel()))
    par = {"rel_l2": rel, "max_abs": float(np.abs(d).max()), "image_max": float(np.abs(xo[:, :, sel]).max()),
           "slices": bounded, "iterations": iters, "bound": PARITY_BOUND, "ok": rel <= PARITY_BOUND,
           "against": "FP64 CPU oracle (oracle/ddfan_oracle.c), same sinogram, from zero"}
    if bounded != pick:
        z = pick[-1]
        par["diverging_slice"] = {
            "slice": z, "oracle_max": float(np.abs(xo[:, :, -1]).max()), "gpu_max": float(np.abs(xg[:, :, z]).max()),
            "why": "slice-0 row sums for every slice and A x kept where a row sum is 0 "
                   "(AAPM_script/OSSART_AAPM.m:63, :88) feed back on this slice's rays"}
    per_iter = secs / iters
    cpu = {"value": 1.0 / (per_iter * s.SLN / len(pick)), "unit": UNIT, "cores": nt, "kind": "port",
           "sample": "%d OS-SART iterations (%d subsets, %d views, FP64, %s) on slices %s of %d, per-iteration "
                     "time scaled by %d/%d (slices are independent); the same run is the parity check"
                     % (iters, s.numOfOS, s.PN, args.back.upper(), pick, s.SLN, s.SLN, len(pick))}
    return par, cpu


def _ossart_host(s, geom, y_h, x_h, out_h, mask, iters, args):
    import ctypes
    from aapm_lowdosectimagerecon_competition_b200._lib import BACK_MODES, SAT_MODES, call
    x0, y0, xds, yds = geom
    hangs = np.ascontiguousarray(view_angles(s, args.views))
    m = np.ascontiguousarray(mask, np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    T = lambda t: ctypes.c_void_p(t.data_ptr())
    call("ddfan_OSSART_AAPM", x0, y0, s.DNU, P(xds), P(yds), s.detCntIdx, 0.0, 0.0, T(y_h), P(hangs),
         s.PN, s.XN, s.YN, s.SLN, s.dx, T(x_h), P(m), iters, s.numOfOS, s.useFISTA, s.nonneg,
         SAT_MODES[args.sat], BACK_MODES[args.back], T(out_h))


def mode_rate(s, geom, y, mask, hangs, sat, back, local, steps=5):
    """OS-SART iterations/s of one solver mode on the bench workload."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import device
    x0, y0, xds, yds = geom
    sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, hangs, s.XN, s.YN, s.SLN, s.dx,
                       mask=mask, numOfOS=s.numOfOS, useFISTA=s.useFISTA, nonneg=s.nonneg,
                       sat=sat, back=back, device=local)
    sv.set_sinogram(y)
    sv.set_image(torch.zeros((s.YN, s.XN, s.SLN), device=y.device))
    st = torch.cuda.current_stream(y.device)
    sv.iterate(2, use_graph=True, stream=st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(y.device)
    e0.record(st)
    sv.iterate(steps, use_graph=True, stream=st)
    e1.record(st)
    torch.cuda.synchronize(y.device)
    sv.close()
    return round(steps / (e0.elapsed_time(e1) / 1e3), 3)


def plain_fp32_iteration(s, geom, y, mask):
    """One OS-SART iteration the way AAPM_script/OSSART_AAPM.m drives the mex
    functions (serve.plain_mex_seconds_per_iter)."""
    from aapm_lowdosectimagerecon_competition_b200 import serve
    sec = serve.plain_mex_seconds_per_iter(s, y.cpu().numpy(), mask)
    return {"value": 1.0 / sec, "unit": UNIT, "seconds_per_iter": sec,
            "how": "mex-style: per subset host->device image, FP32 prefix sums, forward, "
                   "device->host sinogram, host residual, host->device, REF backprojection, "
                   "device->host image, host update (AAPM_script/OSSART_AAPM.m:79-97); no graphs"}


def main():
    args = parse()
    if args.impl == "reference":
        if args.config == "rebin":
            run_rebin_reference(args)
        else:
            run_reference(args)
    elif args.config == "rebin":
        run_rebin(args)
    elif args.kernels:
        run_kernels(args)
    elif args.config == "c2":
        run_c2(args)
    elif args.config == "c4":
        run_c4(args)
    elif args.config == "c5":
        run_c5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
