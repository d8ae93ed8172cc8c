"""ddfan_proj_noalloc: the forward projection for callers that cannot allocate
device memory (their memory belongs to another allocator, or a cudaMalloc's
implicit synchronisation is not acceptable mid-pipeline).  Its scratch is a
fixed device array inside the library.  This file sorts last so that a run
stopping at the first failure has run every other test first; it also passes
on its own in a fresh process.

Each case runs two calls in a row -- a larger problem first, then a smaller
one that lands on the scratch the first left behind -- in every prefix-sum
mode, on a square image and on a rectangular, off-centre one with a slice
count that is not a multiple of 4, and compares each with ddfan_proj_dev on a
plan of the same geometry (same kernels: 1e-6) and with the FP64 oracle (the
parity tolerance of the mode).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SAME = dict(rtol=1e-6, atol=1e-7)  # against ddfan_proj_dev: the same kernels on the same data
ORACLE_TOL = {"fp32": 5e-5, "hilo": 2e-6, "fp64": 2e-6, "direct": 2e-6}
SATS = {"fp32": 0, "hilo": 1, "fp64": 2, "direct": 3}


def _mods():
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import _lib, configs, dd2, device
    from oracle import oracle as O
    assert torch.cuda.is_available()
    return torch, _lib.load(), configs, dd2, device, O


def _case(configs, dd2, shape):
    if shape == "square":
        s = configs.scaled(configs.c2(SLN=8), XN=128, DNU=184, PN=90)
        cx, cy = 0.0, 0.0
    else:
        s = configs.scaled(configs.c2(SLN=7), XN=96, DNU=160, PN=72)
        s.YN = 80
        s.detCntIdx += 0.25
        cx, cy = 3.5, -2.0
    geom = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    return s, geom, np.float32(cx), np.float32(cy)


def _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, mask, sat, stream=None):
    x0, y0, xds, yds = geom
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    st = stream if stream is not None else torch.cuda.current_stream()
    return lib.ddfan_proj_noalloc(x0, y0, s.DNU, P(xds), P(yds), cx, cy, ctypes.c_void_p(angs.data_ptr()),
                                  int(angs.numel()), s.XN, s.YN, s.SLN, ctypes.c_void_p(vol.data_ptr()),
                                  s.dx, None if m is None else P(m), sat, ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_void_p(st.cuda_stream))


def _mask(s):
    yy, xx = np.meshgrid(np.arange(s.YN) - s.YN / 2, np.arange(s.XN) - s.XN / 2, indexing="ij")
    m = ((xx / (0.5 * s.XN)) ** 2 + (yy / (0.5 * s.YN)) ** 2 < 0.85).astype(np.uint8)
    m[:3] = 0
    return m


@pytest.mark.parametrize("sat", sorted(SATS))
@pytest.mark.parametrize("shape", ["square", "rect_offcentre_odd_slices"])
def test_noalloc_matches_plan_and_oracle_on_two_calls(sat, shape):
    torch, lib, configs, dd2, device, O = _mods()
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    # a larger call first (more views, no mask), then the case itself (masked)
    for call in range(2):
        s, geom, cx, cy = _case(configs, dd2, shape)
        if call == 0:
            s.PN *= 2
        mask = _mask(s) if call == 1 else None
        angs_h = s.angles()
        angs = torch.from_numpy(angs_h).cuda()
        vol = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * (0.02 + 0.01 * call)
        x0, y0, xds, yds = geom
        plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx, mask=mask,
                           imgXCenter=cx, imgYCenter=cy, sat=sat)
        ref = plan.proj(angs, vol)
        out = torch.full_like(ref, float("nan"))
        torch.cuda.synchronize()
        rc = _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, mask, SATS[sat])
        assert rc == 0, lib.ddfan_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref.cpu().numpy(), **SAME)
        h = np.repeat(angs_h[:, None], s.SLN, 1)
        exp = O.proj(x0, y0, s.DNU, xds, yds, cx, cy, h, s.PN, s.XN, s.YN, s.SLN, vol.cpu().numpy(), s.dx, mask)
        err = float(np.linalg.norm((got - exp).ravel()) / np.linalg.norm(exp.ravel()))
        assert err < ORACLE_TOL[sat], "call %d: rel-L2 %.3g against the oracle" % (call, err)
        plan.close()


def test_noalloc_allocates_no_device_memory():
    torch, lib, configs, dd2, device, O = _mods()
    s, geom, cx, cy = _case(configs, dd2, "rect_offcentre_odd_slices")
    angs = torch.from_numpy(s.angles()).cuda()
    vol = torch.rand((s.YN, s.XN, s.SLN), device="cuda") * 0.02
    out = torch.empty((s.PN, s.DNU, s.SLN), device="cuda")
    mask = _mask(s)
    for sat in SATS.values():  # warm: module load, first-call set-up
        assert _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, mask, sat) == 0, lib.ddfan_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for sat in SATS.values():
        assert _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, mask, sat) == 0, lib.ddfan_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_refuses_a_capturing_stream():
    torch, lib, configs, dd2, device, O = _mods()
    s, geom, cx, cy = _case(configs, dd2, "square")
    angs = torch.from_numpy(s.angles()).cuda()
    vol = torch.rand((s.YN, s.XN, s.SLN), device="cuda") * 0.02
    out = torch.empty((s.PN, s.DNU, s.SLN), device="cuda")
    assert _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, None, 1) == 0
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(graph, stream=side):
        rcs.append(_noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, None, 1, stream=side))
    assert rcs == [4]  # DDFAN_ERR_UNSUPPORTED, before any CUDA work on the stream
    assert b"captur" in lib.ddfan_last_error()
    # the stream and the scratch still work afterwards
    assert _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, None, 1) == 0
    torch.cuda.synchronize()


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch, lib, configs, dd2, device, O = _mods()
    s, geom, cx, cy = _case(configs, dd2, "square")
    s.XN = s.YN = 1024
    s.SLN = 64
    angs = torch.zeros(8, device="cuda")
    vol = torch.zeros(1, device="cuda")
    out = torch.zeros(1, device="cuda")
    rc = _noalloc(lib, torch, s, geom, cx, cy, angs, vol, out, None, 1)
    assert rc == 4  # DDFAN_ERR_UNSUPPORTED, returned before any GPU work
    assert b"scratch" in lib.ddfan_last_error()
