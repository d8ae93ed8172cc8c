"""Batched OS-SART (ddfan_batch_*): solves of uneven image size, slice count,
view count, subset count, mask and backprojector advanced together with one
launch per kernel kind, subset step and tile class.  Each solve's image must
equal its solo solve bit for bit (the same kernel bodies run with the same
arguments), and match the FP64 oracle.  Needs a B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (side, slices, views, subsets, masked, FISTA, non-negativity, backprojector)
CASES = [(48, 5, 96, 4, True, 1, 1, "adj"), (40, 12, 72, 6, False, 1, 0, "adj"),
         (64, 8, 120, 5, True, 0, 1, "ref"), (32, 33, 90, 3, False, 1, 1, "adj"),
         (56, 17, 60, 4, True, 1, 0, "ref"), (24, 100, 36, 3, True, 1, 1, "ref")]


def _case(configs, dd2, O, N, Z, P, nsub, masked, seed):
    s = configs.scaled(configs.c3(SLN=Z), XN=N, DNU=64, PN=P)
    s.numOfOS = nsub
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = configs.phantom(s, seed=seed)
    mask = s.circular_mask() if masked else None
    y = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, xt, s.dx, mask)
    y = configs.poisson_log(y, 1.5e5, seed=seed)
    return s, (x0, y0, xds, yds), mask, y


@pytest.mark.parametrize("groups", ["1", "3"])
def test_batched_solves_equal_solo_solves_and_oracle(monkeypatch, groups):
    # groups > 1: the solves' launch chains run side by side (graph branches)
    monkeypatch.setenv("DDFAN_BATCH_GROUPS", groups)
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    from oracle import oracle as O
    assert torch.cuda.is_available()
    iters = 3
    cases = [_case(configs, dd2, O, N, Z, P, nsub, m, 20 + i) for i, (N, Z, P, nsub, m, *_r) in enumerate(CASES)]

    def make(i):
        (N, Z, P, nsub, m, fista, nonneg, back) = CASES[i]
        s, (x0, y0, xds, yds), mask, y = cases[i]
        sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, mask=mask,
                           numOfOS=nsub, useFISTA=fista, nonneg=nonneg, sat="direct", back=back)
        sv.set_sinogram(torch.from_numpy(y).cuda())
        sv.set_image(torch.zeros((s.YN, s.XN, s.SLN), device="cuda"))
        return sv

    solo = []
    for i in range(len(CASES)):
        sv = make(i)
        sv.iterate(iters)
        solo.append(sv.image().cpu().numpy())
        sv.close()
    svs = [make(i) for i in range(len(CASES))]
    torch.cuda.synchronize()
    batch = device.OSSARTBatch(svs)
    assert 0 < batch.launches_per_iter < sum(sv.launches_per_iter for sv in svs)
    batch.iterate(1)
    batch.iterate(iters - 1)
    torch.cuda.synchronize()
    for i, sv in enumerate(svs):
        got = sv.image().cpu().numpy()
        np.testing.assert_array_equal(got, solo[i])
        (N, Z, P, nsub, m, fista, nonneg, back) = CASES[i]
        s, (x0, y0, xds, yds), mask, y = cases[i]
        xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, y,
                      np.zeros((s.YN, s.XN, s.SLN), np.float32), s.dx, mask, iters, nsub, fista, nonneg,
                      O.REF if back == "ref" else O.ADJ)
        err = float(np.linalg.norm((got - xo).ravel()) / np.linalg.norm(xo.ravel()))
        assert err < 1e-5, "case %d: rel-L2 %.3g" % (i, err)
    batch.close()
    for sv in svs:
        sv.close()


def test_batch_refuses_table_mode_solvers():
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    from aapm_lowdosectimagerecon_competition_b200._lib import DdfanError
    s = configs.scaled(configs.c3(SLN=4), XN=32, DNU=64, PN=48)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, numOfOS=4,
                       sat="hilo", back="adj")
    with pytest.raises(DdfanError):
        device.OSSARTBatch([sv])
    sv.close()
