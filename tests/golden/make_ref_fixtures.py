"""Generates tests/golden/ref_fixtures.npz from the REFERENCE's own CUDA kernels.

The reference's AAPM_script/MultiSlicesProjGPU.cu and MultiSlicesBackGPU.cu are
compiled unmodified for sm_100a into oracle/_ref/libddref.so (`make -C oracle
ref`, needs the reference tree and nvcc) and driven through their per-GPU host
drivers DD2::DD2_gpu_proj_branchless_sat2d (MultiSlicesProjGPU.cu:211) and
DD2_gpu_back (MultiSlicesBackGPU.cu:187).  This script needs a GPU; it must run
in a process without torch because the reference resets the device on every
call.  It stores, per case, the inputs (so the fixture does not depend on the
phantom code) and the reference's outputs:

    python tests/golden/make_ref_fixtures.py [out.npz]
"""
import ctypes
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFLIB = os.path.join(ROOT, "oracle", "_ref", "libddref.so")


def fan_geometry(sid, sdd, DNU, w, cnt):
    """AAPM_script/DD2MutiSlices.m:55-76 in single precision (1-based channels)."""
    f = np.float32
    step = f(np.arctan(f(f(w) / f(2)) / f(sdd))) * f(2)
    ii = np.arange(1, DNU + 1, dtype=np.float32)
    beta = (ii - f(cnt)) * f(step)
    return (f(0), f(sid), (np.sin(beta) * f(sdd)).astype(f), (f(sid) - np.cos(beta) * f(sdd)).astype(f))


def case_inputs(name, XN, YN, SLN, PN, DNU, dx, sid, sdd, pitch, cnt, cx, cy, per_slice, masked, seed):
    rng = np.random.default_rng(seed)
    x0, y0, xds, yds = fan_geometry(sid, sdd, DNU, pitch, cnt)
    base = np.arange(PN, dtype=np.float64) * (2 * math.pi / PN)
    if per_slice:
        # each slice starts at its own angle (like the rebinned per-slice views)
        off = rng.uniform(0, 2 * math.pi, SLN)
        hangs = (base[:, None] + off[None, :]).astype(np.float32)
    else:
        hangs = np.repeat(base[:, None], SLN, 1).astype(np.float32)
    # smooth positive image: a few random Gaussians on a disk
    yy, xx = np.meshgrid(np.arange(YN) - (YN - 1) / 2, np.arange(XN) - (XN - 1) / 2, indexing="ij")
    vol = np.zeros((YN, XN, SLN), np.float32)
    for z in range(SLN):
        img = np.where(xx ** 2 + yy ** 2 <= (0.45 * min(XN, YN)) ** 2, 0.02, 0.0)
        for _ in range(6):
            c = rng.uniform(-0.3, 0.3, 2) * min(XN, YN)
            s = rng.uniform(0.05, 0.2) * min(XN, YN)
            img = img + rng.uniform(0, 0.03) * np.exp(-((xx - c[0]) ** 2 + (yy - c[1]) ** 2) / (2 * s * s))
        vol[:, :, z] = img
    if masked:
        mask = ((xx / (0.5 * XN)) ** 2 + (yy / (0.5 * YN)) ** 2 < 0.8).astype(np.uint8)
    else:
        mask = np.ones((YN, XN), np.uint8)
    prj_in = rng.uniform(0.0, 1.0, (PN, DNU, SLN)).astype(np.float32)
    return dict(XN=XN, YN=YN, SLN=SLN, PN=PN, DNU=DNU, dx=np.float32(dx), x0=x0, y0=y0, xds=xds, yds=yds,
                detCntIdx=np.float32(cnt), imgXCenter=np.float32(cx), imgYCenter=np.float32(cy),
                hangs=hangs, vol=vol, mask=mask, prj_in=prj_in)


# The reference kernels call __syncthreads() inside per-thread conditions
# (MultiSlicesProjGPU.cu:172,195 after the range check at :118 and the axis
# branch at :152; MultiSlicesBackGPU.cu:181 after the masked early return at
# :131-133).  The cases below keep every thread of every block on the same
# path, so those barriers are uniform: SLN a multiple of 64 (both kernels' x
# block size divides it), DNU a multiple of 8, XN a multiple of 4, one angle
# list for all slices (no per-slice axis switch) and no masked voxels.
CASES = [
    # name, XN, YN, SLN, PN, DNU, dx, sid, sdd, pitch(mm at detector), detCntIdx, imgXCenter,
    # imgYCenter, per-slice angles, masked, seed
    ("siemens32", 32, 32, 64, 36, 64, 11.2, 595.0, 1085.6, 14.79, 32.5, 0.0, 0.0, False, False, 11),
    ("rect_quarter_offcentre", 24, 20, 64, 30, 48, 14.0, 541.0, 949.0, 18.9, 24.75, 3.5, -2.1, False,
     False, 12),
]


def run_reference(c):
    lib = ctypes.CDLL(REFLIB)
    P = ctypes.c_void_p
    f, i = ctypes.c_float, ctypes.c_int
    lib.ddref_proj.argtypes = [f, f, i, P, P, f, f, P, i, i, i, i, P, f, P, P]
    lib.ddref_back.argtypes = [f, f, i, P, P, f, f, f, P, i, i, i, i, P, f, P, P]
    ptr = lambda a: a.ctypes.data_as(P)
    prj = np.zeros((c["PN"], c["DNU"], c["SLN"]), np.float32)
    lib.ddref_proj(c["x0"], c["y0"], c["DNU"], ptr(c["xds"]), ptr(c["yds"]), c["imgXCenter"],
                   c["imgYCenter"], ptr(c["hangs"]), c["PN"], c["XN"], c["YN"], c["SLN"], ptr(c["vol"]),
                   c["dx"], ptr(c["mask"]), ptr(prj))
    vol = np.zeros((c["YN"], c["XN"], c["SLN"]), np.float32)
    lib.ddref_back(c["x0"], c["y0"], c["DNU"], ptr(c["xds"]), ptr(c["yds"]), c["detCntIdx"],
                   c["imgXCenter"], c["imgYCenter"], ptr(c["hangs"]), c["PN"], c["XN"], c["YN"],
                   c["SLN"], ptr(c["prj_in"]), c["dx"], ptr(c["mask"]), ptr(vol))
    return prj, vol


def main(out):
    if not os.path.exists(REFLIB):
        sys.exit("missing %s: run `make -C oracle ref` where the reference tree exists" % REFLIB)
    store = {}
    for spec in CASES:
        name = spec[0]
        c = case_inputs(*spec)
        prj, vol = run_reference(c)
        for k, v in c.items():
            store["%s/%s" % (name, k)] = np.asarray(v)
        store["%s/ref_proj" % name] = prj
        store["%s/ref_back" % name] = vol
        print(name, "proj", float(np.abs(prj).max()), "back", float(np.abs(vol).max()))
    np.savez_compressed(out, **store)
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_fixtures.npz"))
