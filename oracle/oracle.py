"""ctypes front end of the FP64 C oracle (``oracle/ddfan_oracle.c``).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

Function names and argument orders follow the reference's mex entry points:
  ``proj``  <- MultiSlicesProjGPU   (AAPM_script/MultiSlicesProjGPU.cu:550-575)
  ``back``  <- MultiSlicesBackGPU   (AAPM_script/MultiSlicesBackGPU.cu:409-436)
  ``ossart``<- OSSART_AAPM          (AAPM_script/OSSART_AAPM.m:33-118)
Arrays use the C (row-major) view of the MATLAB layouts:
  image    vol[YN][XN][SLN]      (MATLAB single(SLN, XN, YN))
  sinogram prj[PN][DNU][SLN]     (MATLAB single(SLN, DNU, PN))
  angles   hangs[PN][SLN]        (MATLAB single(SLN, PN))
  mask     mask[YN][XN] bytes    (first XN*YN bytes of MATLAB [mask, mask'])
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

REF, ADJ = 0, 1

_f = ctypes.c_float
_i = ctypes.c_int
_p = ctypes.c_void_p


def build():
    """Compile liboracle.so (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_proj.argtypes = [_f, _f, _i, _p, _p, _f, _f, _p, _i, _i, _i, _i, _p, _f, _p, _p, _i]
        L.orc_back.argtypes = [_f, _f, _i, _p, _p, _f, _f, _f, _p, _i, _i, _i, _i, _p, _f, _p, _i,
                               _p, _i]
        L.orc_proj_d.argtypes = L.orc_proj.argtypes
        L.orc_back_d.argtypes = L.orc_back.argtypes
        L.orc_ossart.argtypes = [_f, _f, _i, _p, _p, _f, _f, _f, _p, _i, _i, _i, _i, _p, _p, _f,
                                 _p, _i, _i, _i, _i, _i, _p, _i, _p]
        L.orc_boundaries.argtypes = [_i, _p, _p]
        for fn in (L.orc_proj, L.orc_back, L.orc_proj_d, L.orc_back_d, L.orc_ossart):
            fn.restype = _i
        L.orc_boundaries.restype = None
        _LIB = L
    return _LIB


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _mask(mask, XN, YN):
    if mask is None:
        return np.ones(XN * YN, np.uint8)
    m = _c(mask, np.uint8).reshape(-1)
    assert m.size >= XN * YN
    return m


def nthreads_default():
    return os.cpu_count() or 1


def boundaries(centers):
    c = _c(centers, np.float32)
    out = np.zeros(c.size + 1, np.float64)
    lib().orc_boundaries(c.size, _ptr(c), _ptr(out))
    return out


def proj(x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, hangs, PN, XN, YN, SLN, vol, dx,
         mask=None, nthreads=None, fp64_input=False):
    """FP64 forward projection -> float64 [PN][DNU][SLN]."""
    xds = _c(xds, np.float32); yds = _c(yds, np.float32)
    m = _mask(mask, XN, YN)
    out = np.zeros((PN, DNU, SLN), np.float64)
    nt = nthreads or nthreads_default()
    if fp64_input:
        a = _c(hangs, np.float64); v = _c(vol, np.float64)
        fn = lib().orc_proj_d
    else:
        a = _c(hangs, np.float32); v = _c(vol, np.float32)
        fn = lib().orc_proj
    assert a.size == PN * SLN and v.size == XN * YN * SLN
    rc = fn(x0, y0, DNU, _ptr(xds), _ptr(yds), imgXCenter, imgYCenter, _ptr(a), PN, XN, YN, SLN,
            _ptr(v), dx, _ptr(m), _ptr(out), nt)
    if rc:
        raise RuntimeError("orc_proj failed (%d)" % rc)
    return out


def back(x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PN, XN, YN, SLN, prj,
         dx, mask=None, mode=REF, nthreads=None, fp64_input=False):
    """FP64 backprojection (mode REF or ADJ) -> float64 [YN][XN][SLN]."""
    xds = _c(xds, np.float32); yds = _c(yds, np.float32)
    m = _mask(mask, XN, YN)
    out = np.zeros((YN, XN, SLN), np.float64)
    nt = nthreads or nthreads_default()
    if fp64_input:
        a = _c(hangs, np.float64); q = _c(prj, np.float64)
        fn = lib().orc_back_d
    else:
        a = _c(hangs, np.float32); q = _c(prj, np.float32)
        fn = lib().orc_back
    assert a.size == PN * SLN and q.size == PN * DNU * SLN
    rc = fn(x0, y0, DNU, _ptr(xds), _ptr(yds), detCntIdx, imgXCenter, imgYCenter, _ptr(a), PN,
            XN, YN, SLN, _ptr(q), dx, _ptr(m), int(mode), _ptr(out), nt)
    if rc:
        raise RuntimeError("orc_back failed (%d)" % rc)
    return out


def ossart(x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PNall, XN, YN, SLN,
           proj_meas, init, dx, mask, numOfIter, numOfOS, useFISTA=1, nonneg=0, back_mode=REF,
           nthreads=None, timing=False):
    """FP64 OS-SART (+FISTA, optional non-negativity) -> float64 [YN][XN][SLN]
    (and the iterations' wall time in seconds when timing=True)."""
    xds = _c(xds, np.float32); yds = _c(yds, np.float32)
    a = _c(hangs, np.float32); y = _c(proj_meas, np.float32); x0i = _c(init, np.float32)
    m = _mask(mask, XN, YN)
    out = np.zeros((YN, XN, SLN), np.float64)
    nt = nthreads or nthreads_default()
    secs = ctypes.c_double(0.0)
    rc = lib().orc_ossart(x0, y0, DNU, _ptr(xds), _ptr(yds), detCntIdx, imgXCenter, imgYCenter,
                          _ptr(a), PNall, XN, YN, SLN, _ptr(y), _ptr(x0i), dx, _ptr(m),
                          numOfIter, numOfOS, int(useFISTA), int(nonneg), int(back_mode),
                          _ptr(out), nt, ctypes.byref(secs))
    if rc:
        raise RuntimeError("orc_ossart failed (%d)" % rc)
    return (out, secs.value) if timing else out
