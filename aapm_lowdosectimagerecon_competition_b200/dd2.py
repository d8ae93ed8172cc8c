"""Python mirror of the reference's MATLAB/mex interface for the fan-beam DD path.

Same names, argument order and meaning as the reference, on numpy arrays in the
C (row-major) view of the MATLAB layouts -- the memory is identical:

  MATLAB single(SLN, XN, YN) image     <->  numpy float32 (YN, XN, SLN)
  MATLAB single(SLN, DNU, PN) sinogram <->  numpy float32 (PN, DNU, SLN)
  MATLAB single(SLN, PN) angles        <->  numpy float32 (PN, SLN)
  MATLAB mask(XN, YN)                  <->  numpy uint8   (YN, XN)

Indices (view_ind, startIdx) are 0-based.  Every call runs on the GPU through
libddfan.so; a failure raises DdfanError (the reference prints and exits).

Reference entry points mirrored (paths relative to the reference project root):
  MultiSlicesProjGPU   AAPM_script/MultiSlicesProjGPU.cu:550-575
  MultiSlicesBackGPU   AAPM_script/MultiSlicesBackGPU.cu:409-436
  DD2MutiSlices        AAPM_script/DD2MutiSlices.m:47-117
  OSSART_AAPM          AAPM_script/OSSART_AAPM.m:33-118
  HelicalToFanFunc_mex AAPM_script/HelicalToFanFunc_mex.cpp:186-249 (body :41-185)
  HelicalToFan_routine AAPM_script/HelicalToFan_routine.m:1-45

Raw helical data: MATLAB single(DetHeight, DetWidth, TotalViews) <-> numpy
float32 (TotalViews, DetWidth, DetHeight).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import BACK_MODES, SAT_MODES, call


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _mode(v, table, what):
    if isinstance(v, str):
        try:
            return table[v.lower()]
        except KeyError:
            raise ValueError("unknown %s %r (choose from %s)" % (what, v, sorted(table)))
    return int(v)


def _mask_bytes(mask, XN, YN):
    if mask is None:
        return None
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    if m.size < XN * YN:
        raise ValueError("mask has %d bytes, needs XN*YN = %d" % (m.size, XN * YN))
    return m


def _start_idx(startIdx):
    if startIdx is None:
        return None, 0
    s = np.ascontiguousarray(startIdx, dtype=np.int32).reshape(-1)
    return s, int(s.size)


def fan_geometry(sid, sdd, DNU, detCellWidth, detCntIdx):
    """(x0, y0, xds, yds) as AAPM_script/DD2MutiSlices.m:55-76 builds them
    (1-based channel index, MATLAB single arithmetic)."""
    xds = np.zeros(int(DNU), np.float32)
    yds = np.zeros(int(DNU), np.float32)
    x0 = ctypes.c_float()
    y0 = ctypes.c_float()
    call("ddfan_fan_geometry", sid, sdd, int(DNU), detCellWidth, detCntIdx, ctypes.byref(x0),
         ctypes.byref(y0), _ptr(xds), _ptr(yds))
    return np.float32(x0.value), np.float32(y0.value), xds, yds


def MultiSlicesProjGPU(x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, hangs, PN, XN, YN, SLN, vol,
                       dx, mask=None, startIdx=None, sat="hilo"):
    """Forward projection; returns prj float32 (PN, DNU, SLN)."""
    xds, yds, hangs, vol = _f32(xds), _f32(yds), _f32(hangs), _f32(vol)
    if hangs.size != PN * SLN or vol.size != XN * YN * SLN or xds.size < DNU or yds.size < DNU:
        raise ValueError("array sizes do not match PN/SLN/XN/YN/DNU")
    m = _mask_bytes(mask, XN, YN)
    s, ns = _start_idx(startIdx)
    out = np.empty((PN, DNU, SLN), np.float32)
    call("ddfan_MultiSlicesProjGPU", x0, y0, int(DNU), _ptr(xds), _ptr(yds), imgXCenter, imgYCenter,
         _ptr(hangs), int(PN), int(XN), int(YN), int(SLN), _ptr(vol), dx, _ptr(m), _ptr(s), ns,
         _mode(sat, SAT_MODES, "sat mode"), _ptr(out))
    return out


def MultiSlicesBackGPU(x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PN, XN, YN,
                       SLN, prj, dx, mask=None, startIdx=None, sat="hilo", back="ref"):
    """Backprojection; returns vol float32 (YN, XN, SLN).  back='ref' is the
    reference's backprojector, back='adj' the exact transpose of the forward."""
    xds, yds, hangs, prj = _f32(xds), _f32(yds), _f32(hangs), _f32(prj)
    if hangs.size != PN * SLN or prj.size != PN * DNU * SLN or xds.size < DNU or yds.size < DNU:
        raise ValueError("array sizes do not match PN/SLN/DNU")
    m = _mask_bytes(mask, XN, YN)
    s, ns = _start_idx(startIdx)
    out = np.empty((YN, XN, SLN), np.float32)
    call("ddfan_MultiSlicesBackGPU", x0, y0, int(DNU), _ptr(xds), _ptr(yds), detCntIdx, imgXCenter,
         imgYCenter, _ptr(hangs), int(PN), int(XN), int(YN), int(SLN), _ptr(prj), dx, _ptr(m),
         _ptr(s), ns, _mode(sat, SAT_MODES, "sat mode"), _mode(back, BACK_MODES, "back mode"),
         _ptr(out))
    return out


def _get(cfg, *path):
    v = cfg
    for k in path:
        v = v[k] if isinstance(v, dict) else getattr(v, k)
    return v


def default_start_idx(SLN, numgpu):
    """Slab starts ceil((ii - 1) / numgpu * SLN) of AAPM_script/DD2MutiSlices.m:95-101, 0-based."""
    return np.array([int(np.ceil(ii / numgpu * SLN)) for ii in range(numgpu)], np.int32)


def DD2MutiSlices(flag_fw, cfg, input, hangs, view_ind=None, mask=None, startIdx=None, sat="hilo",
                  back="ref"):
    """AAPM_script/DD2MutiSlices.m:47-117.

    cfg: nested dict/object with recon.{XN, YN, dx}, SLN and
    acq.{sid, sdd, DNU, detCellWidth, detCntIdx}; hangs: (viewNum, SLN) angles;
    view_ind: 0-based views to use (default all); for 'Back', input holds all
    viewNum views and is subset by view_ind as the MATLAB does (:111)."""
    XN, YN = int(_get(cfg, "recon", "XN")), int(_get(cfg, "recon", "YN"))
    dx = np.float32(_get(cfg, "recon", "dx"))
    SLN = int(_get(cfg, "SLN"))
    sid, sdd = np.float32(_get(cfg, "acq", "sid")), np.float32(_get(cfg, "acq", "sdd"))
    DNU = int(_get(cfg, "acq", "DNU"))
    detCntIdx = np.float32(_get(cfg, "acq", "detCntIdx"))
    x0, y0, xds, yds = fan_geometry(sid, sdd, DNU, np.float32(_get(cfg, "acq", "detCellWidth")),
                                    detCntIdx)
    hangs = _f32(hangs).reshape(-1, SLN)
    if view_ind is None:
        view_ind = np.arange(hangs.shape[0])
    view_ind = np.asarray(view_ind, dtype=np.int64).reshape(-1)
    h = _f32(hangs[view_ind])
    PN = int(view_ind.size)
    if mask is None:
        mask = np.ones((YN, XN), np.uint8)
    if startIdx is None:
        startIdx = default_start_idx(SLN, 1)
    if flag_fw == "Proj":
        return MultiSlicesProjGPU(x0, y0, DNU, xds, yds, 0.0, 0.0, h, PN, XN, YN, SLN, input, dx, mask,
                                  startIdx, sat=sat)
    if flag_fw == "Back":
        prj = _f32(input).reshape(-1, DNU, SLN)[view_ind]
        return MultiSlicesBackGPU(x0, y0, DNU, xds, yds, detCntIdx, 0.0, 0.0, h, PN, XN, YN, SLN, prj,
                                  dx, mask, startIdx, sat=sat, back=back)
    raise ValueError("flag_fw must be 'Proj' or 'Back'")


def OSSART_AAPM(Proj, Views, initImg, conf, numOfIter, numOfOS=1, mask=None, useFISTA=1, nonneg=0,
                sat="hilo", back="ref"):
    """AAPM_script/OSSART_AAPM.m:33-118 on the device-resident solver.

    Proj (viewNum, DNU, SLN), Views (viewNum, SLN), initImg (YN, XN, SLN);
    returns the reconstruction float32 (YN, XN, SLN).  Each iteration runs as
    one CUDA graph; nonneg=1 adds a clamp at 0 after every subset update."""
    XN, YN = int(_get(conf, "recon", "XN")), int(_get(conf, "recon", "YN"))
    dx = np.float32(_get(conf, "recon", "dx"))
    Proj = _f32(Proj)
    PNall, DNU, SLN = Proj.shape
    sid, sdd = np.float32(_get(conf, "acq", "sid")), np.float32(_get(conf, "acq", "sdd"))
    detCntIdx = np.float32(_get(conf, "acq", "detCntIdx"))
    x0, y0, xds, yds = fan_geometry(sid, sdd, DNU, np.float32(_get(conf, "acq", "detCellWidth")),
                                    detCntIdx)
    Views = _f32(Views).reshape(PNall, SLN)
    init = _f32(initImg).reshape(YN, XN, SLN)
    m = _mask_bytes(np.ones((YN, XN), np.uint8) if mask is None else mask, XN, YN)
    out = np.empty((YN, XN, SLN), np.float32)
    call("ddfan_OSSART_AAPM", x0, y0, DNU, _ptr(xds), _ptr(yds), detCntIdx, 0.0, 0.0, _ptr(Proj),
         _ptr(Views), PNall, XN, YN, SLN, dx, _ptr(init), _ptr(m), int(numOfIter), int(numOfOS),
         int(useFISTA), int(nonneg), _mode(sat, SAT_MODES, "sat mode"),
         _mode(back, BACK_MODES, "back mode"), _ptr(out))
    return out


def HelicalToFanFunc_mex(proj, zPos, SLN, SD, SO, BVAngle, DetWidth, DetHeight, PerDetW, PerDetH,
                         DefTimes, DetCenterW, SpiralPitchFactor):
    """The mex AAPM_script/HelicalToFanFunc_mex.cpp:186-249 on the GPU.

    proj (TotalViews, DetWidth, DetHeight); returns the mex's layouts
    Proj (SLN, DefTimes, DetWidth) and Views (SLN, DefTimes), bit-identical
    to the reference's CPU result."""
    proj = _f32(proj)
    nViews = int(proj.shape[0])
    if proj.size != nViews * int(DetWidth) * int(DetHeight):
        raise ValueError("proj has %d values, expected TotalViews x DetWidth x DetHeight" % proj.size)
    z = _f32(zPos).reshape(-1)
    SLN = int(SLN)
    if z.size < SLN:
        raise ValueError("zPos has %d entries, SLN = %d" % (z.size, SLN))
    P = np.empty((SLN, int(DefTimes), int(DetWidth)), np.float32)
    V = np.empty((SLN, int(DefTimes)), np.float32)
    call("ddfan_HelicalToFan", _ptr(P), _ptr(V), _ptr(proj), nViews, _ptr(z), SLN, SD, SO, BVAngle,
         int(DetWidth), int(DetHeight), PerDetW, PerDetH, int(DefTimes), DetCenterW, SpiralPitchFactor)
    return P, V


def rebin_params(cfg):
    """The scan constants AAPM_script/HelicalToFan_routine.m:20-33 reads from
    the projection header cfg (nested dict or object; angle in degrees)."""
    return dict(SD=np.float32(_get(cfg, "ConstantRadialDistance")),
                SO=np.float32(_get(cfg, "DetectorFocalCenterRadialDistance")),
                BVAngle=np.float32(_get(cfg, "DetectorFocalCenterAngularPosition") / 180.0 * np.pi),
                DetWidth=int(_get(cfg, "NumberofDetectorColumns")),
                DetHeight=int(_get(cfg, "NumberofDetectorRows")),
                PerDetW=np.float32(_get(cfg, "DetectorElementTransverseSpacing")),
                PerDetH=np.float32(_get(cfg, "DetectorElementAxialSpacing")),
                DefTimes=int(_get(cfg, "NumberofSourceAngularSteps")),
                DetCenterW=np.float32(_get(cfg, "DetectorCentralElement", "X")),
                SpiralPitchFactor=np.float32(_get(cfg, "SpiralPitchFactor")))


def HelicalToFan_routine(proj, cfg, zPos):
    """AAPM_script/HelicalToFan_routine.m:1-45: rebin and permute.

    Returns Proj (DefTimes, DetWidth, SLN) and Views (DefTimes, SLN) -- the
    MATLAB (SLN, DetWidth, DefTimes) and (SLN, DefTimes) arrays, i.e. the
    layouts OSSART_AAPM takes."""
    z = _f32(zPos).reshape(-1)
    P, V = HelicalToFanFunc_mex(proj, z, z.size, **rebin_params(cfg))
    return np.ascontiguousarray(P.transpose(1, 2, 0)), np.ascontiguousarray(V.T)
