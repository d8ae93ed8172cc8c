"""Final-image parity at the workload configurations themselves (not scaled
down), against the FP64 oracle.  Needs a B200.

  c1  256 x 256 x 1 slice, 984 views, 888 channels, sid 541, sdd 949,
      5 OS-SART iterations x 8 subsets with FISTA (OSSART_AAPM.m:33-118),
      the whole reconstruction on both sides.
  c3  512 x 512 x 128, 2304 views, 736 channels, 24 subsets, FISTA and
      non-negativity, Poisson log sinogram at I0 = 1.5e5: the GPU solves all
      128 slices, the oracle two of them (slices are independent given the
      subset weights, which both take from slice 0, OSSART_AAPM.m:61-64).

Bound: relative L2 <= 1e-5 on the final image (the acceptance bound of the
path); the max-abs error is reported in the assertion message.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def errors(got, exp):
    got = np.asarray(got, np.float64)
    d = got - exp
    return float(np.linalg.norm(d.ravel()) / np.linalg.norm(exp.ravel())), float(np.abs(d).max())


@pytest.fixture(scope="module")
def mods():
    import torch
    assert torch.cuda.is_available()
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2
    from oracle import oracle as O
    return configs, dd2, O


@pytest.fixture(scope="module")
def c1_case(mods):
    configs, dd2, O = mods
    s = configs.c1()
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = configs.phantom(s)
    mask = s.circular_mask()
    clean = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, xt, s.dx, mask)
    y = configs.poisson_log(clean, 1.5e5, seed=21)
    init = np.zeros_like(xt)
    xo = {b: O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, y, init,
                      s.dx, mask, s.numOfIter, s.numOfOS, 1, 0, O.REF if b == "ref" else O.ADJ)
          for b in ("ref", "adj")}
    return s, mask, y, init, xo


@pytest.mark.parametrize("sat", ["hilo", "direct", "fp64"])
@pytest.mark.parametrize("back", ["adj", "ref"])
def test_c1_full_reconstruction_matches_oracle(mods, c1_case, sat, back):
    configs, dd2, O = mods
    s, mask, y, init, xo = c1_case
    xg = dd2.OSSART_AAPM(y, s.hangs(), init, s.conf(), s.numOfIter, s.numOfOS, mask, 1, 0, sat=sat, back=back)
    r, m = errors(xg, xo[back])
    assert r <= 1e-5, "c1 %s/%s: rel-L2 %.3g, max-abs %.3g (image max %.3g)" % (sat, back, r, m, xo[back].max())


@pytest.mark.parametrize("sat", ["direct", "hilo"])
def test_c3_full_size_matches_oracle_on_two_slices(mods, sat):
    import torch
    configs, dd2, O = mods
    from aapm_lowdosectimagerecon_competition_b200 import device
    s = configs.c3(SLN=128)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = configs.phantom(s)
    mask = s.circular_mask()
    angs = torch.from_numpy(s.angles()).cuda()
    pl = device.Plan(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.XN, s.YN, s.SLN, s.PN, s.dx, sat="fp64")
    clean = pl.proj(angs, torch.from_numpy(xt).cuda())
    pl.close()
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    counts = torch.poisson(s.I0 * torch.exp(-clean.double()), generator=g)
    y = (-torch.log(torch.clamp(counts, min=1.0) / s.I0)).float()
    iters = 2
    sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, mask=mask,
                       numOfOS=s.numOfOS, useFISTA=1, nonneg=1, sat=sat, back="adj")
    sv.set_sinogram(y)
    sv.set_image(torch.zeros((s.YN, s.XN, s.SLN), device="cuda"))
    sv.iterate(iters)
    xg = sv.image().cpu().numpy()
    sv.close()
    yh = y.cpu().numpy()
    pick = [0, 77]
    ys = np.ascontiguousarray(yh[:, :, pick])
    init = np.zeros((s.YN, s.XN, len(pick)), np.float32)
    h2 = np.ascontiguousarray(s.hangs()[:, :len(pick)])
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h2, s.PN, s.XN, s.YN, len(pick), ys, init, s.dx,
                  mask, iters, s.numOfOS, 1, 1, O.ADJ)
    r, m = errors(xg[:, :, pick], xo)
    assert r <= 1e-5, "c3 %s slices %s: rel-L2 %.3g, max-abs %.3g" % (sat, pick, r, m)
