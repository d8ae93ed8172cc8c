"""Second, independent restatement of the oracle in numpy -- TEST INFRASTRUCTURE.

Written separately from ``ddfan_oracle.c`` (explicit system matrix instead of
prefix-sum tables) so the two can check each other on small cases.  Pure numpy,
meant for images up to ~32x32 and a few dozen views.

Reference formulas followed (paths relative to the reference project root):
  fan_geometry       AAPM_script/DD2MutiSlices.m:49-76 (single precision, 1-based channels)
  boundaries         AAPM_script/utilities.cuh:268-287
  system_matrix      AAPM_script/MultiSlicesProjGPU.cu:100-200 (per-ray footprint per line)
  back_ref           AAPM_script/MultiSlicesBackGPU.cu:115-184, host :187-242
  helical_to_fan     AAPM_script/HelicalToFanFunc_mex.cpp:41-185
"""
import ctypes
import ctypes.util

import numpy as np

TWOPI = 6.283185307179586

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.atanf.restype = ctypes.c_float
_libm.atanf.argtypes = [ctypes.c_float]


def fan_geometry(sid, sdd, DNU, detCellWidth, detCntIdx):
    """Source position and channel centres exactly as DD2MutiSlices.m:55-76
    builds them (MATLAB single arithmetic; channel index ii is 1-based)."""
    f = np.float32
    stepTheta = f(np.arctan(f(f(detCellWidth) / f(2)) / f(sdd))) * f(2)
    ii = np.arange(1, DNU + 1, dtype=np.float32)
    curBeta = (ii - f(detCntIdx)) * f(stepTheta)
    xds = (np.sin(curBeta) * f(sdd)).astype(f)
    yds = (f(sid) - np.cos(curBeta) * f(sdd)).astype(f)
    return f(0.0), f(sid), xds, yds


def boundaries(c):
    c = np.asarray(c, np.float32).astype(np.float64)
    n = c.size + 1
    b = np.empty(n)
    if n >= 3:
        b[0] = 1.5 * c[0] - 0.5 * c[1]
        b[-1] = 1.5 * c[-1] - 0.5 * c[-2]
        b[1:-1] = 0.5 * c[:-1] + 0.5 * c[1:]
    else:
        b[0] = c[0] - 0.5
        b[1] = c[0] + 0.5
    return b.astype(np.float32).astype(np.float64)


def _wrap(a):
    a = float(a)
    while a >= TWOPI:
        a -= TWOPI
    while a < 0:
        a += TWOPI
    return a


def system_matrix(x0, y0, xds, yds, imgXCenter, imgYCenter, angles, XN, YN, dx, mask=None):
    """Single-slice forward operator as a dense matrix A[(p*DNU+u), (y*XN+x)].

    Each row is the reference's ray sum written out pixel by pixel: on every
    line ii the footprint [tL, tR] (texel coords) picks up pixel k with weight
    (ramp(cR, k) - ramp(cL, k)) / len * dx / |dir|, ramp(c, k) = clip(c - k, 0, 1),
    c = clip(t - 0.5, 0, N) -- the same number the padded prefix-sum table
    interpolation gives."""
    x0, y0 = float(x0), float(y0)
    xds = np.asarray(xds, np.float32).astype(np.float64)
    yds = np.asarray(yds, np.float32).astype(np.float64)
    bx, by = boundaries(xds.astype(np.float32)), boundaries(yds.astype(np.float32))
    DNU = xds.size
    ocx = (XN - 1.0) * 0.5 - float(imgXCenter) / float(dx)
    ocy = (YN - 1.0) * 0.5 - float(imgYCenter) / float(dx)
    dx = float(dx)
    PN = len(angles)
    A = np.zeros((PN * DNU, YN * XN))
    for p, th in enumerate(angles):
        th = _wrap(th)
        cs, sn = np.cos(th), np.sin(th)
        sx, sy = x0 * cs - y0 * sn, x0 * sn + y0 * cs
        for u in range(DNU):
            Dx, Dy = xds[u] * cs - yds[u] * sn, xds[u] * sn + yds[u] * cs
            Lx, Ly = bx[u] * cs - by[u] * sn, bx[u] * sn + by[u] * cs
            Rx, Ry = bx[u + 1] * cs - by[u + 1] * sn, bx[u + 1] * sn + by[u + 1] * cs
            d = np.array([Dx - sx, Dy - sy])
            d /= np.hypot(d[0], d[1])
            row = A[p * DNU + u]
            if abs(cs) <= abs(sn):
                fL, fR = (Ly - sy) / (Lx - sx), (Ry - sy) / (Rx - sx)
                cv = dx / abs(d[0])
                N, nl = YN, XN
            else:
                fL, fR = (Lx - sx) / (Ly - sy), (Rx - sx) / (Ry - sy)
                cv = dx / abs(d[1])
                N, nl = XN, YN
            k = np.arange(N)
            for ii in range(nl):
                if abs(cs) <= abs(sn):
                    obj = (ii - ocx) * dx
                    rL, rR = (obj - Lx) * fL + Ly, (obj - Rx) * fR + Ry
                    tL, tR = rL / dx + ocy + 1, rR / dx + ocy + 1
                else:
                    obj = (ii - ocy) * dx
                    rL, rR = (obj - Ly) * fL + Lx, (obj - Ry) * fR + Rx
                    tL, tR = rL / dx + ocx + 1, rR / dx + ocx + 1
                ln = rR - rL
                cL = np.clip(tL - 0.5, 0, N)
                cR = np.clip(tR - 0.5, 0, N)
                w = (np.clip(cR - k, 0, 1) - np.clip(cL - k, 0, 1)) / ln * cv
                if abs(cs) <= abs(sn):
                    row[k * XN + ii] += w
                else:
                    row[ii * XN + k] += w
    if mask is not None:
        m = np.asarray(mask, np.uint8).reshape(-1)[: XN * YN].astype(np.float64)
        A = A * m[None, :]
    return A


def helical_to_fan(proj, zPos, SD, SO, BVAngle, DetWidth, DetHeight, PerDetW, PerDetH, DefTimes,
                   DetCenterW, SpiralPitchFactor):
    """Single-slice helical-to-fan rebinning in the reference's float32
    arithmetic (AAPM_script/HelicalToFanFunc_mex.cpp:41-185).

    proj: raw helical data [TotalViews][DetWidth][DetHeight] (MATLAB
    (Height, Channel, View)).  Returns Proj [DefTimes][DetWidth][SLN] and
    Views [DefTimes][SLN] -- the layouts HelicalToFan_routine.m:44-45 leaves
    after its permutes.  cosf/atanf come from the C library, the functions
    the reference calls, so the result is bit-identical to it on one host."""
    f = np.float32
    proj = np.asarray(proj, np.float32)
    zPos = np.asarray(zPos, np.float32)
    SLN = zPos.size
    SD, SO, BVAngle, PerDetW, PerDetH, DetCenterW, SpiralPitchFactor = (
        f(SD), f(SO), f(BVAngle), f(PerDetW), f(PerDetH), f(DetCenterW), f(SpiralPitchFactor))
    PerDetA = f(2.0) * f(_libm.atanf(float(PerDetW / SD * f(0.5))))      # :160
    delta = f(2.0 * np.pi / DefTimes)                                      # :161
    DetCenterHreal = f((DetHeight - 1.0) * 0.5 / float(PerDetH))           # :162 (divides by PerDetH)
    h = SpiralPitchFactor * PerDetH * f(DetHeight) * SO / SD               # :163
    deltaZ = h / f(DefTimes)                                               # :164
    twopi = f(2.0 * np.pi)
    Proj = np.zeros((DefTimes, DetWidth, SLN), np.float32)
    Views = np.zeros((DefTimes, SLN), np.float32)
    j = np.arange(1, DetWidth + 1)
    ang = (j.astype(np.float32) - DetCenterW) * PerDetA
    SM = SO * np.array([_libm.cosf(float(a)) for a in ang], np.float32)
    for iii in range(SLN):
        z = zPos[iii]
        start = int(np.floor((z - h * f(0.5)) / deltaZ))
        PData = np.zeros((DefTimes, DetWidth), np.float32)
        mark = np.zeros((DefTimes, DetWidth), np.int32)
        angles = np.zeros(DefTimes, np.float32)
        # the reference's loop index is size_t: `i >= start` never holds for
        # start < 0 (the slice stays zero), and i starts at 1 (:73-76)
        first = start + DefTimes if start < 0 else max(1, start)
        for i in range(first, start + DefTimes):
            data = proj[i - 1]                                             # [DetWidth][DetHeight]
            zz = f(i - 1) * deltaZ
            lam = f(i - 1) * delta + BVAngle
            while lam > twopi:                                             # AAPM::mod (:28-34)
                lam = lam - twopi
            ib = i - start                                                 # ibeta - 1
            angles[ib] = lam
            tanAngV = (z - zz) / SM
            v = SD * tanAngV
            dv = (DetCenterHreal + v) / PerDetH + f(1.0)
            idv = np.floor(dv).astype(np.int64)
            t = dv - idv.astype(np.float32)
            cosAngV = SD / np.sqrt(SD * SD + v * v)
            ok = (idv >= 1) & (idv <= DetHeight - 1)
            ii = np.clip(idv, 1, DetHeight - 1)
            d0 = data[j - 1, ii - 1]
            d1 = data[j - 1, ii]
            temp = np.where(ok, d0 * (f(1.0) - t) + d1 * t, f(0.0)).astype(np.float32)
            PData[ib] = cosAngV * temp
            mark[ib] = ok
        bad = (mark == 0).any(axis=1)                                      # :113-123
        PData[bad] = 0
        Proj[:, :, iii] = PData
        Views[:, iii] = angles
    return Proj, Views


def back_ref(x0, y0, xds, yds, detCntIdx, imgXCenter, imgYCenter, angles, XN, YN, dx, prj,
             mask=None):
    """Reference backprojector for one slice: prj[PN][DNU] -> vol[YN][XN]."""
    x0, y0 = float(x0), float(y0)
    xds = np.asarray(xds, np.float32).astype(np.float64)
    yds = np.asarray(yds, np.float32).astype(np.float64)
    DNU = xds.size
    dx = float(dx)
    ocx = (XN - 1.0) * 0.5 - float(imgXCenter) / dx
    ocy = (YN - 1.0) * 0.5 - float(imgYCenter) / dx
    S2D = np.hypot(xds[0] - x0, yds[0] - y0)
    dts = np.hypot(xds[1] - xds[0], yds[1] - yds[0])
    dbeta = np.arctan(dts / S2D * 0.5) * 2.0
    inv_sid = 1.0 / np.hypot(x0, y0)
    iy, ix = np.meshgrid(np.arange(YN), np.arange(XN), indexing="ij")
    vx, vy = (ix - ocx) * dx, (iy - ocy) * dx
    out = np.zeros((YN, XN))
    prj = np.asarray(prj, np.float64)
    for p, th in enumerate(angles):
        th = _wrap(th)
        cs, sn = np.cos(th), np.sin(th)
        sx, sy = x0 * cs - y0 * sn, x0 * sn + y0 * cs
        ddx, ddy = vx - sx, vy - sy
        l2 = ddx * ddx + ddy * ddy
        alpha = np.arcsin((sy * ddx - sx * ddy) * inv_sid / np.sqrt(l2))
        ddv = ddx if abs(sx) > abs(sy) else ddy
        da = ddv / l2 * dx * 0.5
        cosv = dx / ddv * np.sqrt(l2)
        iL = (alpha - da) / dbeta + detCntIdx + 1.0
        iR = (alpha + da) / dbeta + detCntIdx + 1.0
        S = np.concatenate([[0.0], np.cumsum(prj[p])])

        def fetch(t):
            c = np.clip(t - 0.5, 0, DNU)
            i = np.minimum(np.floor(c).astype(int), DNU - 1)
            f = c - i
            return S[i] + f * (S[i + 1] - S[i])

        out += (fetch(iR) - fetch(iL)) * cosv
    if mask is not None:
        m = np.asarray(mask, np.uint8).reshape(-1)[: XN * YN].reshape(YN, XN)
        out = np.where(m != 0, out, 0.0)
    return out
