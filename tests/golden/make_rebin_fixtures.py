"""Generates tests/golden/ref_rebin.npz from the REFERENCE's own CPU rebinning.

The reference's AAPM_script/HelicalToFanFunc_mex.cpp is compiled unmodified
into oracle/_ref/libref_rebin.so (`make -C oracle ref`, needs the reference
tree) and its HelicalToFan (:142-185) is called through the C entry point of
oracle/ref_rebin_harness.cpp.  CPU only.  Each case stores its inputs and the
reference's outputs in the mex layouts Proj (SLN, DefTimes, DetWidth) and
Views (SLN, DefTimes):

    python tests/golden/make_rebin_fixtures.py [out.npz]
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFLIB = os.path.join(ROOT, "oracle", "_ref", "libref_rebin.so")

# name, DetWidth, DetHeight, DefTimes, rotations of raw views, SD, SO, BVAngle (rad),
# PerDetW, PerDetH, DetCenterW, SpiralPitchFactor, seed
CASES = [
    ("siemens_like", 40, 12, 48, 4.5, 1085.6, 595.0, 0.3, 1.2858, 1.0947, 20.25, 0.8, 21),
    ("offcentre_steep", 36, 16, 40, 5.0, 949.0, 541.0, 6.1, 1.40, 1.20, 15.5, 1.4, 22),
]


def z_positions(DefTimes, TotalViews, h, deltaZ):
    """Target slices: the reference's own spread (reconscript.m:22,
    linspace(h, deltaZ * TotalView - h, SLN)) plus edge slices whose
    floor((z - h/2) / deltaZ) is < 0, == 0 and == 1, and one slice that uses
    the very last raw view."""
    inner = np.linspace(h, deltaZ * TotalViews - h, 9)
    edges = [h / 2 - 2.5 * deltaZ, h / 2 + 0.25 * deltaZ, h / 2 + 1.25 * deltaZ,
             (TotalViews - DefTimes + 1) * deltaZ + h / 2 + 0.5 * deltaZ]
    return np.concatenate([edges[:3], inner, edges[3:]]).astype(np.float32)


def run_reference(lib, proj, zPos, SD, SO, BV, W, H, PW, PH, T, CW, pitch):
    SLN = zPos.size
    P = np.zeros((SLN, T, W), np.float32)
    V = np.zeros((SLN, T), np.float32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    # the reference prints one progress line per slice on stdout
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        lib.ddref_helical_to_fan(p(P), p(V), p(proj), p(zPos), SLN, SD, SO, BV, W, H, PW, PH, T, CW, pitch)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    return P, V


def load_reference():
    lib = ctypes.CDLL(REFLIB)
    f, i, v = ctypes.c_float, ctypes.c_int, ctypes.c_void_p
    lib.ddref_helical_to_fan.argtypes = [v, v, v, v, i, f, f, f, i, i, f, f, i, f, f]
    return lib


def main(out):
    lib = load_reference()
    arrays = {}
    for (name, W, H, T, rot, SD, SO, BV, PW, PH, CW, pitch, seed) in CASES:
        rng = np.random.default_rng(seed)
        TV = int(rot * T)
        f = np.float32
        h = f(pitch) * f(PH) * f(H) * f(SO) / f(SD)
        dZ = h / f(T)
        zPos = z_positions(T, TV, float(h), float(dZ))
        proj = (rng.random((TV, W, H)) * 2.0 + 0.5).astype(np.float32)
        P, V = run_reference(lib, proj, zPos, SD, SO, BV, W, H, PW, PH, T, CW, pitch)
        for k, val in dict(proj=proj, zPos=zPos, SD=f(SD), SO=f(SO), BVAngle=f(BV), DetWidth=W, DetHeight=H,
                           PerDetW=f(PW), PerDetH=f(PH), DefTimes=T, DetCenterW=f(CW),
                           SpiralPitchFactor=f(pitch), ref_Proj=P, ref_Views=V).items():
            arrays[name + "/" + k] = np.asarray(val)
        print(name, "raw", proj.shape, "slices", zPos.size, "zeroed rows",
              int((np.abs(P).sum(2) == 0).sum()), file=sys.stderr)
    np.savez_compressed(out, **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_rebin.npz"))
