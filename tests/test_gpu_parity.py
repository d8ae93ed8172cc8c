"""Parity of the sm_100a kernels (through the C ABI) with the FP64 oracle and
with the reference's own kernels.  Needs a B200.

Tolerances (relative L2 against the FP64 oracle):
  compensated hi/lo or FP64 prefix sums, and the direct mode (footprint
  differences summed from the values, no tables): 2e-6 per
  projection/backprojection, 1e-5 on an OS-SART image; plain FP32 prefix sums:
  5e-5 at these sizes.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / np.linalg.norm(np.ravel(b)))


TOL = {"fp32": 5e-5, "hilo": 2e-6, "fp64": 2e-6, "direct": 2e-6}
SATS = ["fp32", "hilo", "fp64", "direct"]


@pytest.fixture(scope="module")
def mods():
    import torch
    assert torch.cuda.is_available()
    from aapm_lowdosectimagerecon_competition_b200 import configs, dd2, device
    from oracle import oracle as O
    return dd2, configs, device, O


def make_case(configs, dd2, XN=40, YN=40, SLN=8, PN=60, DNU=72, cx=0.0, cy=0.0, dcnt=0.0,
              per_slice=False, masked=False, seed=0):
    s = configs.scaled(configs.c2(SLN=SLN), XN=XN, DNU=DNU, PN=PN)
    s.YN = YN
    s.detCntIdx += dcnt
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    rng = np.random.default_rng(seed)
    h = s.hangs()
    if per_slice:
        h = (h + rng.uniform(0, 2 * math.pi, SLN)[None, :]).astype(np.float32)
    vol = (rng.random((YN, XN, SLN)) * 0.03).astype(np.float32)
    mask = None
    if masked:
        yy, xx = np.meshgrid(np.arange(YN) - YN / 2, np.arange(XN) - XN / 2, indexing="ij")
        mask = ((xx / (0.5 * XN)) ** 2 + (yy / (0.5 * YN)) ** 2 < 0.8).astype(np.uint8)
    prj = rng.random((PN, DNU, SLN)).astype(np.float32)
    geo = dict(x0=x0, y0=y0, DNU=DNU, xds=xds, yds=yds, cnt=np.float32(s.detCntIdx),
               cx=np.float32(cx), cy=np.float32(cy), h=h, PN=PN, XN=XN, YN=YN, SLN=SLN,
               dx=np.float32(s.dx), mask=mask)
    return geo, vol, prj


CASES = {
    "square": dict(),
    "rect_offcentre_quarter": dict(XN=36, YN=28, cx=3.5, cy=-2.0, dcnt=0.25),
    "masked_perslice": dict(SLN=5, per_slice=True, masked=True),
    "perslice_rect_odd": dict(SLN=13, XN=36, YN=28, cx=1.5, cy=-2.5, per_slice=True, masked=True),
    "single_slice": dict(SLN=1),
    "odd_slices": dict(SLN=13, XN=24, YN=30),
    "many_slices": dict(SLN=64, XN=32, YN=32, PN=30),
    # 46 float4 slice blocks: two groups of 4 z-tiles of 8 blocks, the second
    # holding 1.75 tiles (partial group and partial tile in the direct kernels)
    "deep_partial_zgroups": dict(SLN=181, XN=20, YN=18, PN=24, masked=True),
}


def fwd(dd2, g, vol, sat):
    return dd2.MultiSlicesProjGPU(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cx"], g["cy"], g["h"],
                                  g["PN"], g["XN"], g["YN"], g["SLN"], vol, g["dx"], g["mask"], sat=sat)


def bwd(dd2, g, prj, sat, back):
    return dd2.MultiSlicesBackGPU(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cnt"], g["cx"], g["cy"],
                                  g["h"], g["PN"], g["XN"], g["YN"], g["SLN"], prj, g["dx"], g["mask"],
                                  sat=sat, back=back)


def ofwd(O, g, vol):
    return O.proj(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cx"], g["cy"], g["h"], g["PN"],
                  g["XN"], g["YN"], g["SLN"], vol, g["dx"], g["mask"])


def obwd(O, g, prj, mode):
    return O.back(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cnt"], g["cx"], g["cy"], g["h"],
                  g["PN"], g["XN"], g["YN"], g["SLN"], prj, g["dx"], g["mask"], mode=mode)


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("sat", SATS)
def test_forward_matches_oracle(mods, case, sat):
    dd2, configs, device, O = mods
    g, vol, _ = make_case(configs, dd2, **CASES[case])
    assert rel(fwd(dd2, g, vol, sat), ofwd(O, g, vol)) < TOL[sat]


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("sat", SATS)
@pytest.mark.parametrize("back", ["ref", "adj"])
def test_backprojection_matches_oracle(mods, case, sat, back):
    dd2, configs, device, O = mods
    g, _, prj = make_case(configs, dd2, **CASES[case])
    out = bwd(dd2, g, prj, sat, back)
    exp = obwd(O, g, prj, O.REF if back == "ref" else O.ADJ)
    assert rel(out, exp) < TOL[sat]
    if g["mask"] is not None:
        assert np.all(out[g["mask"] == 0] == 0)


@pytest.mark.parametrize("sat", ["hilo", "fp64", "direct"])
def test_adjoint_identity_on_gpu(mods, sat):
    dd2, configs, device, O = mods
    g, vol, prj = make_case(configs, dd2, XN=48, YN=40, SLN=8, PN=90, DNU=96, masked=True)
    Ax = fwd(dd2, g, vol, sat).astype(np.float64)
    ATy = bwd(dd2, g, prj, sat, "adj").astype(np.float64)
    lhs, rhs = float((Ax * prj).sum()), float((vol * ATy).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def fixture_cases():
    f = np.load(os.path.join(HERE, "golden", "ref_fixtures.npz"))
    names = sorted({k.split("/")[0] for k in f.files})
    return [(n, {k.split("/", 1)[1]: f[k] for k in f.files if k.startswith(n + "/")}) for n in names]


@pytest.mark.parametrize("name,c", fixture_cases())
def test_ref_mode_matches_reference_kernels(mods, name, c):
    """Drop-in parity with the reference's own kernels (texture precision)."""
    dd2 = mods[0]
    a = (c["x0"], c["y0"], int(c["DNU"]), c["xds"], c["yds"])
    geo = (c["hangs"], int(c["PN"]), int(c["XN"]), int(c["YN"]), int(c["SLN"]))
    P = dd2.MultiSlicesProjGPU(*a, c["imgXCenter"], c["imgYCenter"], *geo, c["vol"], c["dx"], c["mask"])
    assert rel(P, c["ref_proj"]) < 2e-3
    B = dd2.MultiSlicesBackGPU(*a, c["detCntIdx"], c["imgXCenter"], c["imgYCenter"], *geo, c["prj_in"],
                               c["dx"], c["mask"], back="ref")
    assert rel(B, c["ref_back"]) < 2e-3


@pytest.mark.parametrize("threads", ["device", "slab"])
def test_start_idx_slabs_match_single_slab(mods, monkeypatch, threads):
    """Slabs of startIdx equal the one-slab call; with threads=slab every slab
    runs on a host thread of its own (concurrently, here on one GPU)."""
    dd2, configs, device, O = mods
    monkeypatch.setenv("DDFAN_SLAB_THREADS", threads)
    g, vol, prj = make_case(configs, dd2, SLN=11, per_slice=True)
    one = fwd(dd2, g, vol, "hilo")
    args = (g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cx"], g["cy"], g["h"], g["PN"], g["XN"],
            g["YN"], g["SLN"], vol, g["dx"], g["mask"])
    slabs = dd2.MultiSlicesProjGPU(*args, startIdx=[0, 4, 4, 9], sat="hilo")
    np.testing.assert_allclose(slabs, one, rtol=1e-6, atol=1e-7)
    b1 = bwd(dd2, g, prj, "hilo", "adj")
    bs = dd2.MultiSlicesBackGPU(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cnt"], g["cx"], g["cy"],
                                g["h"], g["PN"], g["XN"], g["YN"], g["SLN"], prj, g["dx"], g["mask"],
                                startIdx=dd2.default_start_idx(g["SLN"], 3), back="adj")
    np.testing.assert_allclose(bs, b1, rtol=1e-6, atol=1e-7)
    with pytest.raises(Exception):
        dd2.MultiSlicesProjGPU(*args, startIdx=[1, 4])


@pytest.mark.parametrize("sat", ["hilo", "direct"])
def test_device_api_matches_host_api(mods, sat):
    import torch
    dd2, configs, device, O = mods
    g, vol, prj = make_case(configs, dd2, SLN=12)
    pl = device.Plan(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cnt"], g["XN"], g["YN"], g["SLN"],
                     g["PN"], g["dx"], sat=sat)
    angs = torch.from_numpy(np.ascontiguousarray(g["h"][:, 0])).cuda()
    p_dev = pl.proj(angs, torch.from_numpy(vol).cuda()).cpu().numpy()
    np.testing.assert_allclose(p_dev, fwd(dd2, g, vol, sat), rtol=1e-6, atol=1e-7)
    for back in ("ref", "adj"):
        b_dev = pl.back(angs, torch.from_numpy(prj).cuda(), mode=back).cpu().numpy()
        np.testing.assert_allclose(b_dev, bwd(dd2, g, prj, sat, back), rtol=1e-6, atol=1e-7)
    # per-slice angle tensor (PN, SLN) takes the grouped path
    hp = torch.from_numpy(np.ascontiguousarray(g["h"])).cuda()
    np.testing.assert_allclose(pl.proj(hp, torch.from_numpy(vol).cuda()).cpu().numpy(), p_dev,
                               rtol=1e-6, atol=1e-7)
    pl.close()


def solver_case(configs, dd2, O, SLN=6, XN=40, PN=96, DNU=64, nsub=6):
    s = configs.scaled(configs.c3(SLN=SLN), XN=XN, DNU=DNU, PN=PN)
    s.numOfOS = nsub
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    xt = configs.phantom(s)
    mask = s.circular_mask()
    y = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, xt, s.dx, mask)
    y = configs.poisson_log(y, 1.5e5, seed=5)
    return s, (x0, y0, xds, yds), xt, mask, y


@pytest.mark.parametrize("sat", ["hilo", "direct"])
@pytest.mark.parametrize("back", ["ref", "adj"])
@pytest.mark.parametrize("nonneg", [0, 1])
def test_ossart_matches_oracle(mods, back, nonneg, sat):
    dd2, configs, device, O = mods
    s, (x0, y0, xds, yds), xt, mask, y = solver_case(configs, dd2, O)
    init = np.zeros_like(xt)
    xg = dd2.OSSART_AAPM(y, s.hangs(), init, s.conf(), 5, s.numOfOS, mask, 1, nonneg, sat=sat, back=back)
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, y, init,
                  s.dx, mask, 5, s.numOfOS, 1, nonneg, O.REF if back == "ref" else O.ADJ)
    assert rel(xg, xo) < 1e-5
    if nonneg:
        # the clamp follows every subset update; FISTA's extrapolation after the
        # last subset may dip below 0, so check the clamp without momentum
        x1 = dd2.OSSART_AAPM(y, s.hangs(), init, s.conf(), 2, s.numOfOS, mask, 0, 1, sat=sat, back=back)
        assert x1.min() >= 0


@pytest.mark.parametrize("back", ["ref", "adj"])
@pytest.mark.parametrize("SLN", [5, 8])
def test_direct_solver_masked_initial_image(mods, back, SLN):
    """The direct mode keeps masked voxels at 0 inside the solver and pads the
    slices to a multiple of 4; the image it returns must still be the table
    path's: masked voxels keep their initial value (clamped at 0 by the
    non-negativity step), and FISTA momentum leaves them there."""
    dd2, configs, device, O = mods
    s, (x0, y0, xds, yds), xt, mask, y = solver_case(configs, dd2, O, SLN=SLN)
    rng = np.random.default_rng(11)
    init = (rng.random(xt.shape) * 0.02 - 0.005).astype(np.float32)
    xg = dd2.OSSART_AAPM(y, s.hangs(), init, s.conf(), 3, s.numOfOS, mask, 1, 1, sat="direct", back=back)
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, y, init,
                  s.dx, mask, 3, s.numOfOS, 1, 1, O.REF if back == "ref" else O.ADJ)
    assert rel(xg, xo) < 1e-5
    m0 = mask == 0
    np.testing.assert_array_equal(xg[m0], np.maximum(init[m0], 0))
    xh = dd2.OSSART_AAPM(y, s.hangs(), init, s.conf(), 3, s.numOfOS, mask, 1, 1, sat="hilo", back=back)
    assert rel(xg, xh) < 1e-5


def rebinned_angles(PN, SLN, starts, BV=0.3):
    """Per-slice view angles the way the helical rebinning makes them:
    mod((start_s + ib - 1) * delta + BV, 2 pi) in float32 for slice s, view ib
    (HelicalToFanFunc_mex.cpp:77-81) -- circular shifts of one grid that
    differ from slice to slice in their last bits."""
    f = np.float32
    delta, twopi = f(2 * math.pi / PN), f(2 * math.pi)
    h = np.zeros((PN, SLN), np.float32)
    for z in range(SLN):
        for ib in range(PN):
            lam = f(f(starts[z] + ib) * delta) + f(BV)
            while lam > twopi:
                lam = f(lam - twopi)
            h[ib, z] = lam
    return h


@pytest.mark.parametrize("back,path", [("ref", "auto"), ("ref", "windowed"), ("adj", "auto"), ("adj", "windowed")])
@pytest.mark.parametrize("lists", ["rebinned", "repeating", "unrelated"])
def test_ossart_per_slice_angles_matches_oracle(mods, monkeypatch, back, path, lists):
    """OSSART_AAPM with Views(SLN, PN) that differ per slice (the rebinned
    real-data case): every slice is projected with its own angles and the
    subset weights come from slice 0 (OSSART_AAPM.m:61-64).  Lists that are
    not near-identical windows take the slice-major path by default; the
    windowed path is checked too."""
    dd2, configs, device, O = mods
    if path != "auto":
        monkeypatch.setenv("DDFAN_PER_SLICE", path)
    SLN = 7
    s = configs.scaled(configs.c3(SLN=SLN), XN=40, DNU=64, PN=96)
    s.numOfOS = 6
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    if lists == "rebinned":
        h = rebinned_angles(s.PN, SLN, [37 * z + 5 for z in range(SLN)])
    elif lists == "repeating":
        # three lists over seven slices: A A B C A C C
        base = rebinned_angles(s.PN, 3, [0, 11, 50])
        h = base[:, [0, 0, 1, 2, 0, 2, 2]].copy()
    else:
        # no slice's list is a shifted window of another's
        rng = np.random.default_rng(3)
        h = (s.hangs() + rng.uniform(0, 2 * math.pi, SLN)[None, :].astype(np.float32)).astype(np.float32)
    xt = configs.phantom(s)
    mask = s.circular_mask()
    y = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h, s.PN, s.XN, s.YN, SLN, xt, s.dx, mask)
    y = configs.poisson_log(y, 1.5e5, seed=5)
    init = np.zeros_like(xt)
    xg = dd2.OSSART_AAPM(y, h, init, s.conf(), 4, s.numOfOS, mask, 1, 0, sat="hilo", back=back)
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, s.PN, s.XN, s.YN, SLN, y, init, s.dx, mask, 4,
                  s.numOfOS, 1, 0, O.REF if back == "ref" else O.ADJ)
    assert rel(xg, xo) < 1e-5
    # a slice on its own is the same problem (weights from its own angles
    # only matter for slice 0, which is kept first)
    x_first = dd2.OSSART_AAPM(y[:, :, :1], h[:, :1], init[:, :, :1], dict(s.conf(), SLN=1), 4, s.numOfOS,
                              mask, 1, 0, sat="hilo", back=back)
    assert rel(xg[:, :, :1], x_first) < 1e-6


@pytest.mark.parametrize("sat", ["hilo", "direct"])
def test_ossart_graph_equals_stream_launches(mods, sat):
    import torch
    dd2, configs, device, O = mods
    s, (x0, y0, xds, yds), xt, mask, y = solver_case(configs, dd2, O, SLN=8)
    res = []
    for graph in (True, False):
        sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, s.hangs(), s.XN, s.YN, s.SLN, s.dx, mask=mask,
                           numOfOS=s.numOfOS, useFISTA=1, nonneg=1, sat=sat, back="adj")
        sv.set_sinogram(torch.from_numpy(y).cuda())
        sv.set_image(torch.zeros((s.YN, s.XN, s.SLN)).cuda())
        sv.iterate(3, use_graph=graph)
        torch.cuda.synchronize()
        res.append(sv.image().cpu().numpy())
        sv.close()
    np.testing.assert_array_equal(res[0], res[1])


def test_compensated_sums_beat_fp32_at_full_width(mods):
    """512-pixel lines (config-2 geometry): plain FP32 prefix sums lose accuracy
    in the difference of two large sums; hi/lo and FP64 keep ~1e-7."""
    dd2, configs, device, O = mods
    s = configs.c2(SLN=4)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    PN = 24
    h = np.ascontiguousarray(s.hangs()[::96][:PN])
    vol = configs.ellipsoid_phantom_3d(s)
    exp = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx)
    err = {}
    for sat in ("fp32", "hilo", "fp64", "direct"):
        got = dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx,
                                     sat=sat)
        err[sat] = rel(got, exp)
    assert err["hilo"] < 1e-6 and err["fp64"] < 1e-6 and err["direct"] < 1e-6
    assert err["fp32"] > err["hilo"]


def per_slice_case(configs, dd2, O, SLN=9, XN=40, YN=36, PN=96, DNU=64, nsub=6, seed=5):
    s = configs.scaled(configs.c3(SLN=SLN), XN=XN, DNU=DNU, PN=PN)
    s.YN = YN
    s.numOfOS = nsub
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    # irregular rebinning offsets: residues mod nsub scatter over the slices
    h = rebinned_angles(s.PN, SLN, [int(8.61 * z) + 3 for z in range(SLN)])
    # a centred disk: its chord lengths do not depend on the view angle, so the
    # subset weights of slice 0 (OSSART_AAPM.m:61-64) hold for every slice
    yy, xx = np.meshgrid(np.arange(YN) - (YN - 1) / 2, np.arange(XN) - (XN - 1) / 2, indexing="ij")
    mask = (xx ** 2 + yy ** 2 < (0.45 * min(XN, YN)) ** 2).astype(np.uint8)
    xt = np.ascontiguousarray(configs.phantom(s)[:YN]) * mask[:, :, None]  # the phantom is square: keep YN rows
    y = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h, s.PN, s.XN, s.YN, SLN, xt, s.dx, mask)
    y = configs.poisson_log(y, 1.5e5, seed=seed)
    return s, (x0, y0, xds, yds), h, mask, y


@pytest.mark.parametrize("sat,tol", [("fp32", 1e-4), ("hilo", 1e-5), ("fp64", 1e-5)])
@pytest.mark.parametrize("fista,nonneg", [(1, 0), (0, 1)])
@pytest.mark.parametrize("back", ["adj", "ref"])
def test_slice_major_path_matches_oracle(mods, monkeypatch, sat, tol, fista, nonneg, back):
    """The slice-major path (per-slice geometry, one slice per lane group) in
    every cell format and with both backprojectors, on a rectangular image
    with irregular per-slice lists."""
    dd2, configs, device, O = mods
    monkeypatch.setenv("DDFAN_PER_SLICE", "slices")
    s, (x0, y0, xds, yds), h, mask, y = per_slice_case(configs, dd2, O)
    init = np.zeros((s.YN, s.XN, s.SLN), np.float32)
    xg = dd2.OSSART_AAPM(y, h, init, s.conf(), 3, s.numOfOS, mask, fista, nonneg, sat=sat, back=back)
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, s.PN, s.XN, s.YN, s.SLN, y, init, s.dx, mask, 3,
                  s.numOfOS, fista, nonneg, O.ADJ if back == "adj" else O.REF)
    assert rel(xg, xo) < tol
    if nonneg and not fista:
        assert xg.min() >= 0


def test_slice_major_path_on_shared_angles(mods, monkeypatch):
    """Shared angle lists forced through the slice-major path agree with the
    shared-geometry path (both compensated; different kernels and scan
    orders) and with the oracle."""
    dd2, configs, device, O = mods
    s, (x0, y0, xds, yds), xt, mask, y = solver_case(configs, dd2, O, SLN=9)
    init = np.zeros_like(xt)
    args = (y, s.hangs(), init, s.conf(), 4, s.numOfOS, mask, 1, 1)
    shared = dd2.OSSART_AAPM(*args, sat="hilo", back="adj")
    monkeypatch.setenv("DDFAN_PER_SLICE", "slices")
    sliced = dd2.OSSART_AAPM(*args, sat="hilo", back="adj")
    assert rel(sliced, shared) < 1e-6
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN, y, init, s.dx,
                  mask, 4, s.numOfOS, 1, 1, O.ADJ)
    assert rel(sliced, xo) < 1e-5


def test_slice_major_device_api_and_graphs(mods, monkeypatch):
    """The device solver on the slice-major path: graph and stream launches
    give identical images, and set_image / image round-trip the caller's
    [YN][XN][SLN] layout."""
    import torch
    dd2, configs, device, O = mods
    s, (x0, y0, xds, yds), h, mask, y = per_slice_case(configs, dd2, O, SLN=6)
    res = []
    for graph in (True, False):
        sv = device.OSSART(x0, y0, s.DNU, xds, yds, s.detCntIdx, h, s.XN, s.YN, s.SLN, s.dx, mask=mask,
                           numOfOS=s.numOfOS, useFISTA=1, nonneg=1, sat="hilo", back="adj")
        assert sv.launches_per_iter == s.numOfOS * 7 + 2
        x_in = torch.rand((s.YN, s.XN, s.SLN), device="cuda") * 0.01
        sv.set_image(x_in)
        np.testing.assert_array_equal(sv.image().cpu().numpy(), x_in.cpu().numpy())
        sv.set_sinogram(torch.from_numpy(y).cuda())
        sv.set_image(torch.zeros((s.YN, s.XN, s.SLN)).cuda())
        sv.iterate(3, use_graph=graph)
        torch.cuda.synchronize()
        res.append(sv.image().cpu().numpy())
        sv.close()
    np.testing.assert_array_equal(res[0], res[1])


@pytest.mark.parametrize("back", ["adj", "ref"])
def test_slice_major_uneven_subsets_and_odd_channels(mods, monkeypatch, back):
    """The slice-major solver when the views do not split evenly (98 views in
    5 subsets: 20, 20, 20, 19, 19 -- rows past a short subset's count are
    never read) and the channels do not fill the 31-channel warp groups (61)."""
    dd2, configs, device, O = mods
    monkeypatch.setenv("DDFAN_PER_SLICE", "slices")
    s, (x0, y0, xds, yds), h, mask, y = per_slice_case(configs, dd2, O, SLN=6, XN=34, YN=34, PN=98, DNU=61,
                                                       nsub=5, seed=8)
    init = np.zeros((s.YN, s.XN, s.SLN), np.float32)
    xg = dd2.OSSART_AAPM(y, h, init, s.conf(), 3, s.numOfOS, mask, 1, 0, sat="hilo", back=back)
    xo = O.ossart(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, s.PN, s.XN, s.YN, s.SLN, y, init, s.dx, mask, 3,
                  s.numOfOS, 1, 0, O.ADJ if back == "adj" else O.REF)
    assert rel(xg, xo) < 1e-5


@pytest.mark.parametrize("lists", ["shared", "per_slice"])
def test_slab_sharded_solve_matches_full(mods, monkeypatch, lists):
    """One reconstruction split into the slabs of two ranks (solved one after
    the other here, on one GPU) equals the whole solve: slices are independent
    and, with per-slice lists, each slab solves global slice 0 first for the
    subset weights."""
    from aapm_lowdosectimagerecon_competition_b200 import shard
    dd2, configs, device, O = mods
    if lists == "shared":
        s, (x0, y0, xds, yds), xt, mask, y = solver_case(configs, dd2, O, SLN=9)
        h = s.hangs()
    else:
        monkeypatch.setenv("DDFAN_PER_SLICE", "slices")
        s, (x0, y0, xds, yds), h, mask, y = per_slice_case(configs, dd2, O, SLN=9)
    init = np.zeros((s.YN, s.XN, s.SLN), np.float32)
    kw = dict(mask=mask, numOfOS=s.numOfOS, useFISTA=1, nonneg=1, sat="hilo", back="adj")
    _, _, whole = shard.solve_slab(x0, y0, s.DNU, xds, yds, s.detCntIdx, h, s.XN, s.YN, s.dx, y, init, 3, 0, 1,
                                   **kw)
    parts = [shard.solve_slab(x0, y0, s.DNU, xds, yds, s.detCntIdx, h, s.XN, s.YN, s.dx, y, init, 3, r, 2, **kw)
             for r in range(2)]
    assert [(a, b) for a, b, _ in parts] == [(0, 5), (5, 9)]
    joined = np.concatenate([img.cpu().numpy() for _, _, img in parts], axis=-1)
    assert rel(joined, whole.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("back", ["adj", "ref"])
def test_slice_major_kernels_at_768_pixel_lines(mods, back):
    """The slice-major kernels (taken by per-slice angle lists) at 768-pixel
    lines, where the approximate reciprocal of the footprint length and of the
    bracket width meets the longest lines: projection and backprojection
    within the compensated 2e-6 bound of the FP64 oracle."""
    dd2, configs, device, O = mods
    s = configs.c2(SLN=3)
    s.dx = 0.7 * 512 / 768
    s.XN = s.YN = 768
    PN = 48
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    h = rebinned_angles(2304, 3, [0, 517, 1203])[:PN * 48:48].copy()
    vol = configs.ellipsoid_phantom_3d(s)
    rng = np.random.default_rng(4)
    prj = rng.random((PN, s.DNU, s.SLN)).astype(np.float32)
    got = dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx, sat="hilo")
    exp = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx)
    assert rel(got, exp) < 2e-6
    gb = dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, PN, s.XN, s.YN, s.SLN, prj, s.dx,
                                sat="hilo", back=back)
    eb = O.back(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, PN, s.XN, s.YN, s.SLN, prj, s.dx,
                mode=O.ADJ if back == "adj" else O.REF)
    assert rel(gb, eb) < 2e-6


def test_direct_results_do_not_depend_on_z_tiles_per_thread(mods):
    """The autotuner's second dimension in the direct mode (z-tiles a thread
    walks per decoded footprint, ddfan_tune_set_nz) changes the launch shape
    only: every slice sums the same terms in the same order, so projections
    and both backprojections are bit-identical for 4, 2 and 1."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200._lib import load
    dd2, configs, device, O = mods
    lib = load()
    g, vol, prj = make_case(configs, dd2, SLN=150, XN=36, YN=30, PN=40, masked=True)
    zb = (g["SLN"] + 3) // 4
    angs = torch.from_numpy(np.ascontiguousarray(g["h"][:, 0])).cuda()
    vt, pt = torch.from_numpy(vol).cuda(), torch.from_numpy(prj).cuda()
    outs = {}
    try:
        for nz in (4, 2, 1):
            assert lib.ddfan_tune_set_nz(zb, nz) == 0
            assert lib.ddfan_tune_get_nz(zb) == nz
            pl = device.Plan(g["x0"], g["y0"], g["DNU"], g["xds"], g["yds"], g["cnt"], g["XN"], g["YN"],
                             g["SLN"], g["PN"], g["dx"], mask=g["mask"], sat="direct")
            outs[nz] = [pl.proj(angs, vt).cpu().numpy(), pl.back(angs, pt, mode="adj").cpu().numpy(),
                        pl.back(angs, pt, mode="ref").cpu().numpy()]
            pl.close()
    finally:
        lib.ddfan_tune_set_nz(zb, 0)
    for nz in (2, 1):
        for a, b in zip(outs[4], outs[nz]):
            np.testing.assert_array_equal(a, b)
    assert rel(outs[4][0], ofwd(O, g, vol)) < TOL["direct"]


@pytest.mark.parametrize("N", [768, 1024])
def test_direct_kernels_at_long_lines(mods, N):
    """The direct mode sums each ray in one FP32 running sum over its lines
    (no chunk sums): at the longest lines a plan takes (1024 pixels) the
    projection and both backprojections stay within the 2e-6 bound of the
    FP64 oracle."""
    dd2, configs, device, O = mods
    s = configs.c2(SLN=8)
    s.dx = 0.7 * 512 / N
    s.XN = s.YN = N
    PN = 24
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    h = np.repeat(s.angles(PN)[:, None], s.SLN, 1).astype(np.float32)
    vol = configs.ellipsoid_phantom_3d(s)
    prj = np.random.default_rng(8).random((PN, s.DNU, s.SLN)).astype(np.float32)
    got = dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx, sat="direct")
    exp = O.proj(x0, y0, s.DNU, xds, yds, 0, 0, h, PN, s.XN, s.YN, s.SLN, vol, s.dx)
    assert rel(got, exp) < 2e-6
    for back, mode in (("adj", O.ADJ), ("ref", O.REF)):
        gb = dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, PN, s.XN, s.YN, s.SLN, prj,
                                    s.dx, sat="direct", back=back)
        eb = O.back(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, h, PN, s.XN, s.YN, s.SLN, prj, s.dx, mode=mode)
        assert rel(gb, eb) < 2e-6
