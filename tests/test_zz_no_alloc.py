"""ddfan_proj_noalloc: the forward projection for callers that cannot allocate
device memory (their memory belongs to another allocator, or a cudaMalloc's
implicit synchronisation is not acceptable mid-pipeline).  Its scratch is a
fixed device array inside the library.  This file sorts last so that a run
stopping at the first failure has run every other test first; it also passes
on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-6, atol=1e-7)  # the hi/lo tolerance of the parity tests


def _setup():
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2
    assert torch.cuda.is_available()
    s = configs.scaled(configs.c2(SLN=8), XN=128, DNU=184, PN=90)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    return torch, s, (x0, y0, xds, yds)


def _noalloc(lib, torch, s, geom, angs, vol, out, mask=None, sat=1):
    x0, y0, xds, yds = geom
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    return lib.ddfan_proj_noalloc(x0, y0, s.DNU, P(xds), P(yds), 0.0, 0.0, ctypes.c_void_p(angs.data_ptr()),
                                  int(angs.numel()), s.XN, s.YN, s.SLN, ctypes.c_void_p(vol.data_ptr()),
                                  s.dx, None if m is None else P(m), sat, ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_plan_projection_twice():
    torch, s, geom = _setup()
    from aapm_lowdosectimagerecon_competition_b200 import _lib, device
    lib = _lib.load()
    x0, y0, xds, yds = geom
    angs = torch.from_numpy(s.angles()).cuda()
    mask = s.circular_mask()
    mask[:5] = 0
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    for call, (sat, use_mask) in enumerate([(1, False), (1, True)]):
        vol = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * (0.02 + 0.01 * call)
        plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx,
                           mask=mask if use_mask else None, sat="hilo")
        ref = plan.proj(angs, vol)
        out = torch.full_like(ref, float("nan"))
        rc = _noalloc(lib, torch, s, geom, angs, vol, out, mask if use_mask else None, sat)
        assert rc == 0, lib.ddfan_last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), **TOL)
        plan.close()


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch, s, geom = _setup()
    from aapm_lowdosectimagerecon_competition_b200 import _lib
    lib = _lib.load()
    big = s
    big.XN = big.YN = 1024
    big.SLN = 64
    angs = torch.zeros(8, device="cuda")
    vol = torch.zeros(1, device="cuda")
    out = torch.zeros(1, device="cuda")
    rc = _noalloc(lib, torch, big, geom, angs, vol, out)
    assert rc == 4  # DDFAN_ERR_UNSUPPORTED, returned before any GPU work
    assert b"scratch" in lib.ddfan_last_error()
