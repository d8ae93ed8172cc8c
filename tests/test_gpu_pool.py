"""The library's device memory pool: memory of a destroyed plan stays in it
for the next plan (no new mapping per solve) until ddfan_release_cached."""
import gc

import pytest

pytestmark = pytest.mark.gpu


def test_pool_keeps_freed_memory_until_released():
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    assert torch.cuda.is_available()
    s = configs.scaled(configs.c2(SLN=16), XN=256, DNU=368, PN=180)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    gc.collect()
    device.release_cached(0)
    base = device.cached_bytes(0)  # partly used blocks of live objects may stay
    mk = lambda: device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx, sat="hilo")
    plan = mk()
    held = plan.device_bytes
    plan.close()
    torch.cuda.synchronize()
    kept = device.cached_bytes(0)
    assert kept >= base + held // 2
    again = mk()  # served from the kept blocks
    torch.cuda.synchronize()
    assert device.cached_bytes(0) <= kept - held // 2
    again.close()
    device.release_cached(0)
    assert device.cached_bytes(0) <= base
