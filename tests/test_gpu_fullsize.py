"""Properties of the sm_100a path at the full OS-SART size (512 x 512 x 128
image, 736 channels, 2304 views in 24 subsets of 96), where the FP64 oracle
would take hours: adjoint consistency, linearity, views past one launch's
grid, and a descending OS-SART residual.  Needs a B200.

Tolerances: <A x, y> against <x, A^T y> to 1e-6 (relative); linearity of the
projector and the exact-adjoint backprojector to 2e-6 relative L2 (the
per-projection tolerance of the compensated hi/lo cells)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full():
    import torch
    assert torch.cuda.is_available()
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    s = configs.c3()
    geom = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    return torch, s, geom, device


def subset_angles(torch, s, k=5):
    # subset k of the interleaved 24-subset split (views k, k + 24, ...)
    return torch.from_numpy(np.ascontiguousarray(s.angles()[k::s.numOfOS])).cuda()


def dot64(a, b):
    return float((a.double() * b.double()).sum())


def rel(a, b):
    return float((a.double() - b.double()).norm() / b.double().norm())


@pytest.mark.parametrize("sat", ["hilo", "fp64"])
def test_adjoint_identity_full_size(full, sat):
    torch, s, (x0, y0, xds, yds), device = full
    angs = subset_angles(torch, s)
    plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, angs.numel(), s.dx,
                       mask=s.circular_mask(), sat=sat)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * 0.02
    y = torch.rand((angs.numel(), s.DNU, s.SLN), device="cuda", generator=g)
    lhs = dot64(plan.proj(angs, x), y)
    rhs = dot64(x, plan.back(angs, y, mode="adj"))
    plan.close()
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_linearity_full_size(full):
    torch, s, (x0, y0, xds, yds), device = full
    angs = subset_angles(torch, s, k=17)
    plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, angs.numel(), s.dx, sat="hilo")
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    a, b = 0.75, -1.5
    x = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * 0.02
    z = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * 0.02
    exp = a * plan.proj(angs, x).double() + b * plan.proj(angs, z).double()
    assert rel(plan.proj(angs, a * x + b * z), exp) < 2e-6
    p = torch.rand((angs.numel(), s.DNU, s.SLN), device="cuda", generator=g)
    q = torch.rand((angs.numel(), s.DNU, s.SLN), device="cuda", generator=g)
    exp = a * plan.back(angs, p).double() + b * plan.back(angs, q).double()
    assert rel(plan.back(angs, a * p + b * q), exp) < 2e-6
    plan.close()


def test_views_beyond_one_grid_are_projected(full):
    """70000 views in one call: the projector launches views past the 65535
    grid rows in a second launch; every view equals its projection in a call
    of its own range (views are independent, so bit for bit)."""
    torch, s, (x0, y0, xds, yds), device = full
    XN = YN = 64
    SLN, PN = 4, 70000
    g = torch.Generator(device="cuda")
    g.manual_seed(13)
    angs = torch.rand(PN, device="cuda", generator=g) * (2 * np.pi)
    vol = torch.rand((YN, XN, SLN), device="cuda", generator=g) * 0.02
    plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, XN, YN, SLN, PN, 5.0, sat="hilo")
    full_prj = plan.proj(angs, vol)
    torch.cuda.synchronize()
    for lo, hi in ((0, 900), (65000, 66200), (PN - 700, PN)):
        part = plan.proj(angs[lo:hi].contiguous(), vol)
        assert torch.equal(full_prj[lo:hi], part), (lo, hi)
    assert bool(torch.isfinite(full_prj).all()) and float(full_prj.abs().sum()) > 0
    plan.close()


@pytest.mark.parametrize("useFISTA", [0, 1])
def test_ossart_residual_descends_full_size(full, useFISTA):
    """Two full-size OS-SART iterations (24 subsets, non-negativity, one CUDA
    graph per iteration) from zero on noiseless data: the data residual falls
    below a quarter of |y|.  Without momentum the image is non-negative; with
    it the extrapolation after each iteration's clamp may dip below zero,
    as in the reference's update order."""
    torch, s, (x0, y0, xds, yds), device = full
    from aapm_lowdosectimagerecon_competition_b200 import configs
    xt = torch.from_numpy(configs.ellipsoid_phantom_3d(s)).cuda()
    mask = s.circular_mask()
    angs = torch.from_numpy(s.angles()).cuda()
    plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx, mask=mask, sat="hilo")
    y = plan.proj(angs, xt)
    sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, mask=mask,
                       numOfOS=s.numOfOS, useFISTA=useFISTA, nonneg=1, sat="hilo", back="adj")
    sv.set_sinogram(y)
    sv.set_image(torch.zeros_like(xt))
    sv.iterate(2)
    img = sv.image()
    torch.cuda.synchronize()
    sv.close()
    assert bool(torch.isfinite(img).all())
    if not useFISTA:
        assert float(img.min()) >= 0.0
    r = rel(plan.proj(angs, img), y)
    plan.close()
    assert r < 0.25, r


def test_per_slice_lists_full_size(full):
    """Per-slice angle lists (helical rebinning, slices 86.07 raw views apart;
    one 96-view subset of every slice's window) through the plan at full
    size: the slice-major forward and exact adjoint satisfy the adjoint
    identity to 1e-6, and a slice's projection matches a one-slice
    shared-list projection of that slice with its own list."""
    torch, s, (x0, y0, xds, yds), device = full
    hp_all = s.rebinned_hangs(spacing=86.07)
    hp = np.ascontiguousarray(hp_all[5::s.numOfOS])  # (96, 128), every slice its own list
    PN = hp.shape[0]
    mask = s.circular_mask()
    plan = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, PN, s.dx, mask=mask, sat="hilo")
    g = torch.Generator(device="cuda")
    g.manual_seed(14)
    x = torch.rand((s.YN, s.XN, s.SLN), device="cuda", generator=g) * 0.02
    y = torch.rand((PN, s.DNU, s.SLN), device="cuda", generator=g)
    ha = torch.from_numpy(hp).cuda()
    Ax = plan.proj(ha, x)
    lhs = dot64(Ax, y)
    rhs = dot64(x, plan.back(ha, y, mode="adj"))
    assert abs(lhs - rhs) / abs(lhs) < 1e-6
    one = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, 1, PN, s.dx, mask=mask, sat="hilo")
    for z in (0, 77, 127):
        az = torch.from_numpy(np.ascontiguousarray(hp[:, z])).cuda()
        ref = one.proj(az, x[:, :, z:z + 1].contiguous())
        assert rel(Ax[:, :, z:z + 1], ref) < 1e-6, z
    one.close()
    plan.close()
