"""The MATLAB mex shims (aapm_lowdosectimagerecon_competition_b200/mex/*.c)
compiled against a stand-in of the mex API (tests/fakemex/) and called the way
MATLAB calls them: argument checks on CPU, results equal to the library's
entry points on the GPU."""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "aapm_lowdosectimagerecon_competition_b200")
SHIMS = ("MultiSlicesProjGPU", "MultiSlicesBackGPU", "HelicalToFanFunc_mex")
SINGLE, INT32, UINT8, DOUBLE = 7, 12, 9, 6


class Mex:
    """One compiled shim plus the fake API's helpers."""

    def __init__(self, path):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.fm_wrap.restype = ctypes.c_void_p
        L.fm_wrap.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
        L.fm_data.restype = ctypes.c_void_p
        L.fm_data.argtypes = [ctypes.c_void_p]
        L.fm_numel.restype = ctypes.c_size_t
        L.fm_numel.argtypes = [ctypes.c_void_p]
        L.fm_free.argtypes = [ctypes.c_void_p]
        L.fm_call.restype = ctypes.c_int
        L.fm_call.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_char_p, ctypes.c_size_t]

    def call(self, nlhs, args):
        """args: (numpy array, class id); numpy C arrays are MATLAB arrays with reversed dims."""
        keep, ptrs = [], []
        for a, cls in args:
            a = np.ascontiguousarray(a)
            keep.append(a)
            dims = (ctypes.c_size_t * max(1, a.ndim))(*(reversed(a.shape) if a.ndim else (1,)))
            ptrs.append(self.lib.fm_wrap(cls, max(1, a.ndim), dims, a.ctypes.data_as(ctypes.c_void_p)))
        prhs = (ctypes.c_void_p * len(ptrs))(*ptrs)
        plhs = (ctypes.c_void_p * max(1, nlhs))()
        msg = ctypes.create_string_buffer(512)
        fn = ctypes.cast(self.lib.mexFunction, ctypes.c_void_p)
        rc = self.lib.fm_call(fn, nlhs, plhs, len(ptrs), prhs, msg, 512)
        for p in ptrs:
            self.lib.fm_free(p)
        if rc:
            return None, msg.value.decode()
        outs = []
        for i in range(nlhs):
            n = self.lib.fm_numel(plhs[i])
            buf = (ctypes.c_float * n).from_address(self.lib.fm_data(plhs[i]))
            outs.append(np.array(buf, dtype=np.float32))
            self.lib.fm_free(plhs[i])
        return outs, None


@pytest.fixture(scope="module")
def shims(tmp_path_factory):
    from aapm_lowdosectimagerecon_competition_b200 import _lib
    _lib.load()
    d = tmp_path_factory.mktemp("mex")
    out = {}
    for name in SHIMS:
        so = str(d / ("%s.so" % name))
        subprocess.run(["gcc", "-std=c99", "-O1", "-fPIC", "-shared", "-Wall", "-Werror",
                        "-I" + os.path.join(HERE, "fakemex"), "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(PKG, "mex"), os.path.join(PKG, "mex", name + ".c"),
                        os.path.join(HERE, "fakemex", "fakemex.c"), "-L" + PKG, "-lddfan",
                        "-Wl,-rpath," + PKG, "-o", so], check=True)
        out[name] = Mex(so)
    return out


def f32(x):
    return (np.asarray(x, np.float32), SINGLE)


def i32(x):
    return (np.asarray(x, np.int32), INT32)


def proj_args(SLN=4, PN=12, DNU=40, XN=24, seed=0):
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2
    s = configs.scaled(configs.c2(SLN=SLN), XN=XN, DNU=DNU, PN=PN)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    rng = np.random.default_rng(seed)
    h = (s.hangs() + rng.uniform(0, 2 * math.pi, SLN)[None, :]).astype(np.float32)
    vol = rng.random((XN, XN, SLN)).astype(np.float32)
    prj = rng.random((PN, DNU, SLN)).astype(np.float32)
    mask = np.ones((XN, XN), np.uint8)
    return s, (x0, y0, xds, yds), h, vol, prj, mask


def test_shims_build_and_check_their_arguments(shims):
    out, err = shims["MultiSlicesProjGPU"].call(1, [f32(0.0)] * 3)
    assert out is None and "16 inputs" in err
    out, err = shims["MultiSlicesBackGPU"].call(1, [f32(0.0)] * 16)
    assert out is None and "17 inputs" in err
    out, err = shims["HelicalToFanFunc_mex"].call(2, [f32(0.0)] * 12)
    assert out is None and "13 inputs" in err
    # a double where the reference passes single (DD2MutiSlices.m casts with single())
    s, (x0, y0, xds, yds), h, vol, prj, mask = proj_args()
    args = [f32(x0), f32(y0), i32(s.DNU), f32(xds), f32(yds), f32(0), f32(0), f32(h), i32(s.PN), i32(s.XN),
            i32(s.YN), i32(s.SLN), (vol.astype(np.float64), DOUBLE), f32(s.dx), (mask, UINT8), i32([0])]
    out, err = shims["MultiSlicesProjGPU"].call(1, args)
    assert out is None and "input 13 must be single" in err


def test_shim_without_a_gpu_raises_the_library_error(shims):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s, (x0, y0, xds, yds), h, vol, prj, mask = proj_args()
    args = [f32(x0), f32(y0), i32(s.DNU), f32(xds), f32(yds), f32(0), f32(0), f32(h), i32(s.PN), i32(s.XN),
            i32(s.YN), i32(s.SLN), f32(vol), f32(s.dx), (mask, UINT8), i32([0])]
    out, err = shims["MultiSlicesProjGPU"].call(1, args)
    assert out is None and err


@pytest.mark.gpu
def test_proj_and_back_shims_equal_the_library(shims):
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    s, (x0, y0, xds, yds), h, vol, prj, mask = proj_args()
    args = [f32(x0), f32(y0), i32(s.DNU), f32(xds), f32(yds), f32(0), f32(0), f32(h), i32(s.PN), i32(s.XN),
            i32(s.YN), i32(s.SLN), f32(vol), f32(s.dx), (mask, UINT8), i32([0])]
    out, err = shims["MultiSlicesProjGPU"].call(1, args)
    assert err is None
    exp = dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h, s.PN, s.XN, s.YN, s.SLN, vol, s.dx, mask,
                                 sat="hilo")
    np.testing.assert_array_equal(out[0].reshape(exp.shape), exp)
    for back in ("ref", "adj"):
        os.environ["DDFAN_MEX_BACK"] = back
        try:
            bargs = [f32(x0), f32(y0), i32(s.DNU), f32(xds), f32(yds), f32(s.detCntIdx), f32(0), f32(0), f32(h),
                     i32(s.PN), i32(s.XN), i32(s.YN), i32(s.SLN), f32(prj), f32(s.dx), (mask, UINT8), i32([0])]
            out, err = shims["MultiSlicesBackGPU"].call(1, bargs)
        finally:
            del os.environ["DDFAN_MEX_BACK"]
        assert err is None
        exp = dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, s.PN, s.XN, s.YN, s.SLN, prj,
                                     s.dx, mask, sat="hilo", back=back)
        np.testing.assert_array_equal(out[0].reshape(exp.shape), exp)


@pytest.mark.gpu
def test_rebinning_shim_equals_the_reference_fixture(shims):
    f = np.load(os.path.join(HERE, "golden", "ref_rebin.npz"))
    name = sorted({k.split("/")[0] for k in f.files})[0]
    c = {k.split("/", 1)[1]: f[k] for k in f.files if k.startswith(name + "/")}
    z = c["zPos"]
    args = [f32(c["proj"]), f32(z), i32(z.size), f32(c["SD"]), f32(c["SO"]), f32(c["BVAngle"]),
            i32(c["DetWidth"]), i32(c["DetHeight"]), f32(c["PerDetW"]), f32(c["PerDetH"]), i32(c["DefTimes"]),
            f32(c["DetCenterW"]), f32(c["SpiralPitchFactor"])]
    out, err = shims["HelicalToFanFunc_mex"].call(2, args)
    assert err is None
    np.testing.assert_array_equal(out[0].reshape(c["ref_Proj"].shape), c["ref_Proj"])
    np.testing.assert_array_equal(out[1].reshape(c["ref_Views"].shape), c["ref_Views"])
