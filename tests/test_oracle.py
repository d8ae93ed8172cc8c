"""The FP64 oracle, pinned against the reference's own kernels and checked
against an independent numpy restatement and analytic answers (CPU only)."""
import math
import os

import numpy as np
import pytest

from oracle import np_oracle as N
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_fixtures.npz")


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / np.linalg.norm(np.ravel(b)))


def fixture_cases():
    f = np.load(FIX)
    names = sorted({k.split("/")[0] for k in f.files})
    return [(n, {k.split("/", 1)[1]: f[k] for k in f.files if k.startswith(n + "/")}) for n in names]


def small_geometry(XN=12, YN=12, DNU=32, PN=16, SLN=3, cnt=None, sid=541.0, sdd=949.0, pitch=20.0,
                   per_slice=False, seed=0):
    rng = np.random.default_rng(seed)
    cnt = (DNU + 1) / 2 if cnt is None else cnt
    x0, y0, xds, yds = N.fan_geometry(sid, sdd, DNU, pitch, cnt)
    a = np.arange(PN) * 2 * math.pi / PN
    if per_slice:
        h = (a[:, None] + rng.uniform(0, 2 * math.pi, SLN)[None, :]).astype(np.float32)
    else:
        h = np.repeat(a[:, None], SLN, 1).astype(np.float32)
    return x0, y0, xds, yds, np.float32(cnt), h


# ------------------------------------------------------------ reference pins

@pytest.mark.parametrize("name,c", fixture_cases())
def test_oracle_matches_reference_kernels(name, c):
    """Oracle vs the reference's own CUDA kernels (tests/golden/make_ref_fixtures.py).
    The reference samples its prefix sums with hardware linear filtering
    (8-bit fractional weights) and FP32 sums, so agreement is at ~1e-3."""
    args = (c["x0"], c["y0"], int(c["DNU"]), c["xds"], c["yds"])
    geo = (c["hangs"], int(c["PN"]), int(c["XN"]), int(c["YN"]), int(c["SLN"]))
    P = O.proj(*args, c["imgXCenter"], c["imgYCenter"], *geo, c["vol"], c["dx"], c["mask"])
    assert rel(P, c["ref_proj"]) < 2e-3
    B = O.back(*args, c["detCntIdx"], c["imgXCenter"], c["imgYCenter"], *geo, c["prj_in"], c["dx"],
               c["mask"], mode=O.REF)
    assert rel(B, c["ref_back"]) < 2e-3
    # the exact adjoint is a different operator from the reference's backprojector
    Ba = O.back(*args, c["detCntIdx"], c["imgXCenter"], c["imgYCenter"], *geo, c["prj_in"],
                c["dx"], c["mask"], mode=O.ADJ)
    assert rel(Ba, c["ref_back"]) > 0.1


# ------------------------------------------------------------ restatements

@pytest.mark.parametrize("XN,YN,per_slice,masked,cx,cy,dcnt", [
    (12, 12, False, False, 0.0, 0.0, 0.0),
    (10, 14, True, True, 3.0, -2.0, 0.25),
    (16, 9, False, True, -1.5, 0.7, -0.3),
])
def test_c_oracle_matches_numpy_restatement(XN, YN, per_slice, masked, cx, cy, dcnt):
    DNU, PN, SLN = 32, 16, 3
    cx, cy = np.float32(cx), np.float32(cy)  # the C entry points take float arguments
    x0, y0, xds, yds, cnt, h = small_geometry(XN, YN, DNU, PN, SLN, cnt=(DNU + 1) / 2 + dcnt,
                                              per_slice=per_slice)
    rng = np.random.default_rng(1)
    vol = rng.random((YN, XN, SLN)).astype(np.float32)
    prj = rng.random((PN, DNU, SLN)).astype(np.float32)
    mask = (rng.random((YN, XN)) > 0.3).astype(np.uint8) if masked else None
    dx = np.float32(20.0)
    P = O.proj(x0, y0, DNU, xds, yds, cx, cy, h, PN, XN, YN, SLN, vol, dx, mask)
    Bref = O.back(x0, y0, DNU, xds, yds, cnt, cx, cy, h, PN, XN, YN, SLN, prj, dx, mask, mode=O.REF)
    Badj = O.back(x0, y0, DNU, xds, yds, cnt, cx, cy, h, PN, XN, YN, SLN, prj, dx, mask, mode=O.ADJ)
    for z in range(SLN):
        A = N.system_matrix(x0, y0, xds, yds, cx, cy, h[:, z], XN, YN, dx, mask)
        np.testing.assert_allclose(P[:, :, z].ravel(), A @ vol[:, :, z].ravel().astype(np.float64),
                                   rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(Badj[:, :, z].ravel(), A.T @ prj[:, :, z].ravel().astype(np.float64),
                                   rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(Bref[:, :, z], N.back_ref(x0, y0, xds, yds, cnt, cx, cy, h[:, z], XN, YN,
                                                             dx, prj[:, :, z], mask), rtol=1e-10, atol=1e-12)


def test_adjoint_identity():
    x0, y0, xds, yds, cnt, h = small_geometry(20, 20, 40, 24, 2)
    rng = np.random.default_rng(2)
    vol = rng.random((20, 20, 2)).astype(np.float32)
    prj = rng.random((24, 40, 2)).astype(np.float32)
    P = O.proj(x0, y0, 40, xds, yds, 0, 0, h, 24, 20, 20, 2, vol, 20.0)
    B = O.back(x0, y0, 40, xds, yds, cnt, 0, 0, h, 24, 20, 20, 2, prj, 20.0, mode=O.ADJ)
    lhs, rhs = float((P * prj).sum()), float((vol * B).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_reference_back_is_one_bin_off_the_transpose():
    """Regression marker: the reference backprojector adds +1 to a 1-based
    detCntIdx (MultiSlicesBackGPU.cu:175-176) and so sits one channel off the
    transpose of the forward; shifting detCntIdx by -1 brings it close."""
    XN = YN = 12
    DNU, PN = 32, 16
    x0, y0, xds, yds, cnt, h = small_geometry(XN, YN, DNU, PN, 1, pitch=2.0 * 1.0239, sdd=949.0)
    a = h[:, 0]
    A = N.system_matrix(x0, y0, xds, yds, 0, 0, a, XN, YN, 1.0)

    def bmat(c):
        cols = []
        for j in range(PN * DNU):
            e = np.zeros(PN * DNU)
            e[j] = 1
            cols.append(N.back_ref(x0, y0, xds, yds, c, 0, 0, a, XN, YN, 1.0, e.reshape(PN, DNU)).ravel())
        return np.stack(cols, 1)

    nA = np.linalg.norm(A)
    assert np.linalg.norm(bmat(cnt) - A.T) / nA > 0.5
    assert np.linalg.norm(bmat(cnt - 1) - A.T) / nA < 0.02


# ------------------------------------------------------------ analytic pins

def test_row_sums_are_chord_lengths_over_dx():
    """A 1 (no mask) equals the geometric length of each channel's central ray
    inside the image square divided by dx -- the reference's forward carries a
    1/dx factor (prefix sums in pixel units over lengths in mm)."""
    XN = YN = 24
    dx = np.float32(10.0)
    DNU, PN = 64, 8
    x0, y0, xds, yds, cnt, h = small_geometry(XN, YN, DNU, PN, 1, pitch=6.0)
    P = O.proj(x0, y0, DNU, xds, yds, 0, 0, h, PN, XN, YN, 1, np.ones((YN, XN, 1), np.float32), dx)
    half = XN * float(dx) / 2
    for p in range(PN):
        th = float(h[p, 0])
        c, s = math.cos(th), math.sin(th)
        src = np.array([x0 * c - y0 * s, x0 * s + y0 * c])
        for u in range(0, DNU, 7):
            d = np.array([xds[u] * c - yds[u] * s, xds[u] * s + yds[u] * c]) - src
            d /= np.linalg.norm(d)
            # slab intersection with [-half, half]^2
            t0, t1 = -1e18, 1e18
            for k in range(2):
                if abs(d[k]) < 1e-15:
                    continue
                a, b = (-half - src[k]) / d[k], (half - src[k]) / d[k]
                t0, t1 = max(t0, min(a, b)), min(t1, max(a, b))
            L = max(0.0, t1 - t0)
            # DD smears the ray over its footprint: near-edge rays differ
            if L > 0.3 * XN * float(dx):
                assert abs(P[p, u, 0] - L / float(dx)) < 0.02 * L / float(dx)


def test_disk_projection_is_analytic():
    """Uniform disk: DD forward ~ mu * chord / dx (loose; DD blurs by one footprint)."""
    XN = YN = 64
    dx = np.float32(4.0)
    R = 90.0
    mu = 0.02
    c = (np.arange(XN) - (XN - 1) / 2) * float(dx)
    X, Y = np.meshgrid(c, c)
    vol = np.where(X ** 2 + Y ** 2 <= R ** 2, mu, 0.0).astype(np.float32)[:, :, None]
    DNU, PN = 96, 6
    x0, y0, xds, yds, cnt, h = small_geometry(XN, YN, DNU, PN, 1, pitch=4.0)
    P = O.proj(x0, y0, DNU, xds, yds, 0, 0, h, PN, XN, YN, 1, vol, dx)
    for p in range(PN):
        th = float(h[p, 0])
        cs, sn = math.cos(th), math.sin(th)
        src = np.array([x0 * cs - y0 * sn, x0 * sn + y0 * cs])
        for u in range(10, DNU - 10, 5):
            d = np.array([xds[u] * cs - yds[u] * sn, xds[u] * sn + yds[u] * cs]) - src
            d /= np.linalg.norm(d)
            dist = abs(src[0] * d[1] - src[1] * d[0])
            if dist < 0.8 * R:
                chord = 2 * math.sqrt(R * R - dist * dist)
                assert abs(P[p, u, 0] - mu * chord / float(dx)) < 0.05 * mu * chord / float(dx)


def test_slices_are_independent():
    x0, y0, xds, yds, cnt, h = small_geometry(14, 14, 30, 12, 4, per_slice=True)
    vol = np.random.default_rng(3).random((14, 14, 4)).astype(np.float32)
    P = O.proj(x0, y0, 30, xds, yds, 0, 0, h, 12, 14, 14, 4, vol, 20.0)
    for z in range(4):
        Pz = O.proj(x0, y0, 30, xds, yds, 0, 0, np.ascontiguousarray(h[:, z:z + 1]), 12, 14, 14, 1,
                    np.ascontiguousarray(vol[:, :, z:z + 1]), 20.0)
        np.testing.assert_allclose(P[:, :, z], Pz[:, :, 0], rtol=1e-14, atol=0)


def test_ossart_reduces_residual():
    XN = YN = 16
    DNU, PN, SLN = 40, 40, 2
    x0, y0, xds, yds, cnt, h = small_geometry(XN, YN, DNU, PN, SLN, pitch=12.0)
    rng = np.random.default_rng(4)
    xt = rng.random((YN, XN, SLN)).astype(np.float32) * 0.02
    dx = np.float32(15.0)
    y = O.proj(x0, y0, DNU, xds, yds, 0, 0, h, PN, XN, YN, SLN, xt, dx).astype(np.float32)
    res = []
    for it in (1, 4):
        x = O.ossart(x0, y0, DNU, xds, yds, cnt, 0, 0, h, PN, XN, YN, SLN, y, np.zeros_like(xt), dx, None,
                     it, 4, 1, 0, O.ADJ)
        Px = O.proj(x0, y0, DNU, xds, yds, 0, 0, h, PN, XN, YN, SLN, x.astype(np.float32), dx)
        res.append(rel(Px, y))
    assert res[1] < res[0] < 1.0


def test_fan_geometry_restatement_matches_matlab_formula():
    x0, y0, xds, yds = N.fan_geometry(595.0, 1085.6, 736, 1.2858, 368.5)
    step = 2 * math.atan(1.2858 / 2 / 1085.6)
    beta = (np.arange(1, 737) - 368.5) * step
    np.testing.assert_allclose(xds, 1085.6 * np.sin(beta), rtol=0, atol=2e-4)
    np.testing.assert_allclose(yds, 595.0 - 1085.6 * np.cos(beta), rtol=0, atol=2e-4)
    assert x0 == 0 and y0 == np.float32(595.0)


def test_reference_update_diverges_with_per_slice_lists():
    """A finding about the reference's OS-SART, not about the kernels: it takes
    slice 0's row and column sums for every slice (OSSART_AAPM.m:63-64) and
    keeps A x where a row sum is 0 (:88).  With one angle list per slice (as
    rebinning makes them) a rotated slice has rays that cross the masked disk
    where slice 0's rays miss it, and those rays feed the image back into
    itself: one iteration takes slice 77 to ~80x the phantom's maximum while
    slice 0 stays bounded, for both backprojectors.  The solvers reproduce
    this, so per-slice parity is bounded on slice 0."""
    from aapm_lowdosectimagerecon_competition_b200 import configs
    s = configs.scaled(configs.c3(SLN=128), XN=64, PN=576, DNU=184)
    s.numOfOS = 8
    x0, y0, xds, yds = N.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    hs = np.ascontiguousarray(s.rebinned_hangs(spacing=86.07 * 576 / 2304)[:, [0, 77]])
    xt = np.ascontiguousarray(configs.phantom(s)[:, :, [0, 77]])
    y = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, hs, s.PN, s.XN, s.YN, 2, xt, s.dx, None).astype(np.float32)
    for back in (O.REF, O.ADJ):
        x = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0.0, 0.0, hs, s.PN, s.XN, s.YN, 2, y,
                     np.zeros_like(xt), s.dx, s.circular_mask(), 1, s.numOfOS, 1, 1, back_mode=back, nthreads=4)
        top = np.abs(x).reshape(-1, 2).max(0)
        assert top[0] < 1.5 * xt.max()
        assert top[1] > 20 * xt.max()
