"""Device-resident API on torch CUDA tensors (plans and the OS-SART solver).

Torch supplies device memory and streams only; all compute runs in
libddfan.so kernels.  Tensors use the reference layouts (see dd2.py).
"""
import ctypes

import numpy as np
import torch

from ._lib import BACK_MODES, SAT_MODES, call, load
from .dd2 import _f32, _mask_bytes, _mode, _ptr


def _dptr(t):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
        raise ValueError("expected a contiguous CUDA tensor")
    if t.dtype != torch.float32:
        raise ValueError("expected float32, got %s" % t.dtype)
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def cached_bytes(device=None):
    """Device bytes the library's memory pool holds unused (freed by
    destroyed plans and solvers, kept for the next ones)."""
    d = torch.cuda.current_device() if device is None else int(device)
    return int(load().ddfan_cached_bytes(d))


def release_cached(device=None):
    """Return the pool's unused device memory to the driver (synchronises
    the device)."""
    d = torch.cuda.current_device() if device is None else int(device)
    call("ddfan_release_cached", d)


class Plan:
    """Geometry + scratch for repeated projections of one shape
    (ddfan_plan_create; replaces the per-call set-up of the reference's
    DD2_gpu_proj_branchless_sat2d / DD2_gpu_back)."""

    def __init__(self, x0, y0, DNU, xds, yds, detCntIdx, XN, YN, SLN, PNmax, dx, mask=None,
                 imgXCenter=0.0, imgYCenter=0.0, sat="hilo", device=None):
        load()
        self.DNU, self.XN, self.YN, self.SLN, self.PNmax = int(DNU), int(XN), int(YN), int(SLN), int(PNmax)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        xds, yds = _f32(xds), _f32(yds)
        m = _mask_bytes(mask, XN, YN)
        h = ctypes.c_void_p()
        call("ddfan_plan_create", ctypes.byref(h), x0, y0, self.DNU, _ptr(xds), _ptr(yds), detCntIdx,
             imgXCenter, imgYCenter, self.XN, self.YN, dx, _ptr(m), self.SLN, self.PNmax,
             _mode(sat, SAT_MODES, "sat mode"), self.device.index)
        self._h = h

    @property
    def device_bytes(self):
        return int(load().ddfan_plan_device_bytes(self._h))

    def proj(self, angs, vol, out=None, stream=None):
        """angs: (PN,) shared or (PN, SLN) per-slice device angles; vol (YN, XN, SLN)."""
        PN = angs.shape[0]
        per_slice = 1 if angs.dim() == 2 else 0
        if out is None:
            out = torch.empty((PN, self.DNU, self.SLN), device=vol.device, dtype=torch.float32)
        call("ddfan_proj_dev", self._h, _dptr(angs), PN, per_slice, _dptr(vol), _dptr(out), _stream(stream))
        return out

    def back(self, angs, prj, out=None, mode="adj", stream=None):
        PN = angs.shape[0]
        per_slice = 1 if angs.dim() == 2 else 0
        if out is None:
            out = torch.empty((self.YN, self.XN, self.SLN), device=prj.device, dtype=torch.float32)
        call("ddfan_back_dev", self._h, _dptr(angs), PN, per_slice, _dptr(prj), _dptr(out),
             _mode(mode, BACK_MODES, "back mode"), _stream(stream))
        return out

    def close(self):
        if getattr(self, "_h", None):
            load().ddfan_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OSSART:
    """Device-resident OS-SART/FISTA solve (ddfan_ossart_*): the measured
    sinogram, the image, the FISTA state, the weights and the per-view tables
    stay on the GPU; each iteration is one CUDA graph replay."""

    def __init__(self, x0, y0, DNU, xds, yds, detCntIdx, hangs, XN, YN, SLN, dx, mask=None,
                 numOfOS=1, useFISTA=1, nonneg=0, sat="hilo", back="adj", imgXCenter=0.0,
                 imgYCenter=0.0, device=None):
        load()
        hangs = _f32(hangs).reshape(-1, SLN)
        self.PNall, self.DNU, self.XN, self.YN, self.SLN = hangs.shape[0], int(DNU), int(XN), int(YN), int(SLN)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        m = _mask_bytes(mask, XN, YN)
        h = ctypes.c_void_p()
        call("ddfan_ossart_create", ctypes.byref(h), x0, y0, self.DNU, _ptr(_f32(xds)), _ptr(_f32(yds)),
             detCntIdx, imgXCenter, imgYCenter, _ptr(hangs), self.PNall, self.XN, self.YN, self.SLN, dx,
             _ptr(m), int(numOfOS), int(useFISTA), int(nonneg), _mode(sat, SAT_MODES, "sat mode"),
             _mode(back, BACK_MODES, "back mode"), self.device.index)
        self._h = h

    @property
    def device_bytes(self):
        return int(load().ddfan_ossart_device_bytes(self._h))

    @property
    def launches_per_iter(self):
        return int(load().ddfan_ossart_launches_per_iter(self._h))

    def set_sinogram(self, proj, stream=None):
        if isinstance(proj, torch.Tensor) and proj.is_cuda:
            call("ddfan_ossart_set_sinogram", self._h, _dptr(proj), 1, _stream(stream))
        else:
            a = _f32(proj)
            if isinstance(proj, torch.Tensor):
                a = _f32(proj.numpy())
            call("ddfan_ossart_set_sinogram", self._h, a.ctypes.data_as(ctypes.c_void_p), 0,
                 _stream(stream))

    def set_image(self, img, stream=None):
        if isinstance(img, torch.Tensor) and img.is_cuda:
            call("ddfan_ossart_set_image", self._h, _dptr(img), 1, _stream(stream))
        else:
            a = _f32(img.numpy() if isinstance(img, torch.Tensor) else img)
            call("ddfan_ossart_set_image", self._h, a.ctypes.data_as(ctypes.c_void_p), 0, _stream(stream))

    def iterate(self, n, use_graph=True, stream=None):
        call("ddfan_ossart_iterate", self._h, int(n), 1 if use_graph else 0, _stream(stream))

    def image(self, out=None, stream=None):
        """Copy of the current image as a CUDA tensor (YN, XN, SLN)."""
        if out is None:
            out = torch.empty((self.YN, self.XN, self.SLN), device=self.device, dtype=torch.float32)
        call("ddfan_ossart_get_image", self._h, _dptr(out), 1, _stream(stream))
        return out

    def image_host(self, out=None, stream=None):
        if out is None:
            out = np.empty((self.YN, self.XN, self.SLN), np.float32)
        ptr = out.ctypes.data_as(ctypes.c_void_p) if isinstance(out, np.ndarray) else ctypes.c_void_p(out.data_ptr())
        call("ddfan_ossart_get_image", self._h, ptr, 0, _stream(stream))
        return out

    KINDS = ("view_geom", "sat_image", "fwd", "sat_sino", "back_a", "back_b", "fista")

    def profile(self, n=1, stream=None):
        """Device ms and launch count per kernel kind over n ungraphed iterations."""
        ms = (ctypes.c_float * 7)()
        cnt = (ctypes.c_int * 7)()
        call("ddfan_ossart_profile", self._h, int(n), _stream(stream), ms, cnt)
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KINDS)}

    def close(self):
        if getattr(self, "_h", None):
            load().ddfan_ossart_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OSSARTBatch:
    """Many device-resident OS-SART solves advanced together
    (ddfan_batch_*): every iteration runs each solve's next iteration with one
    launch per kernel kind, subset step and tile class over all of them.  The
    solvers (OSSART objects in the direct mode, one angle list each) must
    outlive the batch; set their sinograms and images first."""

    def __init__(self, solvers):
        load()
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[sv._h.value for sv in self.solvers])
        h = ctypes.c_void_p()
        call("ddfan_batch_create", ctypes.byref(h), arr, len(self.solvers))
        self._h = h

    @property
    def launches_per_iter(self):
        return int(load().ddfan_batch_launches_per_iter(self._h))

    def iterate(self, n, use_graph=True, stream=None):
        call("ddfan_batch_iterate", self._h, int(n), 1 if use_graph else 0, _stream(stream))

    def close(self):
        if getattr(self, "_h", None):
            load().ddfan_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
