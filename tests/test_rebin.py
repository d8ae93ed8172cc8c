"""Helical-to-fan rebinning: the restatement pinned bit-for-bit to the
reference's CPU code, the GPU kernels bit-for-bit to the restatement."""
import ctypes
import os

import numpy as np
import pytest

from oracle import np_oracle as N

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = os.path.join(HERE, "golden", "ref_rebin.npz")
REFLIB = os.path.join(ROOT, "oracle", "_ref", "libref_rebin.so")

SCALARS = ("SD", "SO", "BVAngle", "DetWidth", "DetHeight", "PerDetW", "PerDetH", "DefTimes", "DetCenterW",
           "SpiralPitchFactor")


def fixture_cases():
    f = np.load(FIX)
    names = sorted({k.split("/")[0] for k in f.files})
    return [(n, {k.split("/", 1)[1]: f[k] for k in f.files if k.startswith(n + "/")}) for n in names]


def params(c):
    out = {}
    for k in SCALARS:
        v = c[k]
        out[k] = int(v) if k in ("DetWidth", "DetHeight", "DefTimes") else np.float32(v)
    return out


def oracle_mex_layout(proj, zPos, p):
    P, V = N.helical_to_fan(proj, zPos, **p)
    return np.ascontiguousarray(P.transpose(2, 0, 1)), np.ascontiguousarray(V.T)


def synthetic(W=48, H=16, T=60, rot=4.4, SD=1085.6, SO=595.0, BV=0.3, PW=1.2858, PH=1.0947, CW=24.5,
              pitch=1.0, SLN=23, seed=0, edges=True):
    f = np.float32
    rng = np.random.default_rng(seed)
    TV = int(rot * T)
    h = f(pitch) * f(PH) * f(H) * f(SO) / f(SD)
    dZ = h / f(T)
    z = np.linspace(float(h), float(dZ) * TV - float(h), SLN)
    if edges:
        z = np.concatenate([[float(h) / 2 - 1.5 * float(dZ), float(h) / 2 + 0.5 * float(dZ)], z])
    proj = (rng.random((TV, W, H)) + 0.25).astype(np.float32)
    p = dict(SD=f(SD), SO=f(SO), BVAngle=f(BV), DetWidth=W, DetHeight=H, PerDetW=f(PW), PerDetH=f(PH), DefTimes=T,
             DetCenterW=f(CW), SpiralPitchFactor=f(pitch))
    return proj, z.astype(np.float32), p


# ------------------------------------------------------------ CPU: restatement pins

@pytest.mark.parametrize("name,c", fixture_cases())
def test_restatement_matches_reference_fixture(name, c):
    """numpy restatement vs the reference's own HelicalToFan (fixture made by
    tests/golden/make_rebin_fixtures.py): identical bits, zeroed rows included."""
    P, V = oracle_mex_layout(c["proj"], c["zPos"], params(c))
    np.testing.assert_array_equal(P, c["ref_Proj"])
    np.testing.assert_array_equal(V, c["ref_Views"])
    # the cases exercise every row rule: a start < 0 slice (all zero), a start == 0
    # slice (view 0 zero), rows zeroed because a channel leaves the detector
    zero_rows = (np.abs(c["ref_Proj"]).sum(2) == 0)
    assert zero_rows[0].all() and zero_rows[1, 0] and not zero_rows[1, 1:].all()


@pytest.mark.skipif(not os.path.exists(REFLIB), reason="reference rebinning not compiled (make -C oracle ref)")
@pytest.mark.parametrize("seed,pitch,CW", [(3, 0.6, 24.5), (4, 1.5, 30.25)])
def test_restatement_matches_reference_library(seed, pitch, CW):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_rebin_fixtures as M
    proj, z, p = synthetic(pitch=pitch, CW=CW, seed=seed)
    ref_P, ref_V = M.run_reference(M.load_reference(), proj, z, p["SD"], p["SO"], p["BVAngle"], p["DetWidth"],
                                   p["DetHeight"], p["PerDetW"], p["PerDetH"], p["DefTimes"], p["DetCenterW"],
                                   p["SpiralPitchFactor"])
    P, V = oracle_mex_layout(proj, z, p)
    np.testing.assert_array_equal(P, ref_P)
    np.testing.assert_array_equal(V, ref_V)


def test_view_angles_are_one_rotation_shifted():
    """Per-slice angles are mod((i - 1) delta + BVAngle, 2 pi) over one rotation
    of raw views i (HelicalToFanFunc_mex.cpp:77-81)."""
    proj, z, p = synthetic(SLN=5, edges=False)
    _, V = N.helical_to_fan(proj, z, **p)
    T = p["DefTimes"]
    d = np.diff(V.astype(np.float64), axis=0) % (2 * np.pi)
    assert np.allclose(d, 2 * np.pi / T, atol=1e-5)
    assert (V >= 0).all() and (V <= np.float32(2 * np.pi)).all()


def test_host_rejects_out_of_range_slices():
    """A slice whose rotation of raw views runs past the data is an argument
    error (the reference reads past its buffer); checked before any GPU work."""
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    from aapm_lowdosectimagerecon_competition_b200._lib import DdfanError
    proj, z, p = synthetic(SLN=4, edges=False)
    T = p["DefTimes"]
    f = np.float32
    h = f(p["SpiralPitchFactor"]) * f(p["PerDetH"]) * f(p["DetHeight"]) * f(p["SO"]) / f(p["SD"])
    bad = np.array([z[0], float(h / f(T)) * (proj.shape[0] + 3)], np.float32)
    with pytest.raises(DdfanError) as e:
        dd2.HelicalToFanFunc_mex(proj, bad, 2, **p)
    assert e.value.code == 1 and "raw view" in str(e.value)


def test_rebin_params_from_header_cfg():
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    cfg = dict(ConstantRadialDistance=1085.6, DetectorFocalCenterRadialDistance=595.0,
               DetectorFocalCenterAngularPosition=90.0, NumberofDetectorColumns=736, NumberofDetectorRows=64,
               DetectorElementTransverseSpacing=1.2858, DetectorElementAxialSpacing=1.0947,
               NumberofSourceAngularSteps=2304, DetectorCentralElement=dict(X=369.625), SpiralPitchFactor=0.8)
    p = dd2.rebin_params(cfg)
    assert p["DetWidth"] == 736 and p["DefTimes"] == 2304
    assert p["BVAngle"] == np.float32(np.pi / 2) and p["DetCenterW"] == np.float32(369.625)


# ------------------------------------------------------------ GPU parity

@pytest.mark.gpu
@pytest.mark.parametrize("name,c", fixture_cases())
def test_gpu_rebin_matches_reference_fixture(name, c):
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    p = params(c)
    P, V = dd2.HelicalToFanFunc_mex(c["proj"], c["zPos"], c["zPos"].size, **p)
    np.testing.assert_array_equal(P, c["ref_Proj"])
    np.testing.assert_array_equal(V, c["ref_Views"])


@pytest.mark.gpu
@pytest.mark.parametrize("SLN,pitch,seed", [(23, 1.0, 0), (70, 1.5, 1), (1, 0.7, 2)])
def test_gpu_rebin_routine_and_device_layouts(SLN, pitch, seed):
    """HelicalToFan_routine (permuted layouts) and the device entry in both
    layouts, SLN not a multiple of 32, against the restatement."""
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    from aapm_lowdosectimagerecon_competition_b200._lib import call
    proj, z, p = synthetic(SLN=SLN, pitch=pitch, seed=seed, edges=SLN > 1)
    oP, oV = N.helical_to_fan(proj, z, **p)
    cfg = dict(ConstantRadialDistance=p["SD"], DetectorFocalCenterRadialDistance=p["SO"],
               DetectorFocalCenterAngularPosition=float(p["BVAngle"]) * 180.0 / np.pi,
               NumberofDetectorColumns=p["DetWidth"], NumberofDetectorRows=p["DetHeight"],
               DetectorElementTransverseSpacing=p["PerDetW"], DetectorElementAxialSpacing=p["PerDetH"],
               NumberofSourceAngularSteps=p["DefTimes"], DetectorCentralElement=dict(X=p["DetCenterW"]),
               SpiralPitchFactor=p["SpiralPitchFactor"])
    q = dd2.rebin_params(cfg)
    if q["BVAngle"] != p["BVAngle"]:  # degrees round trip: use the angle the routine will use
        p["BVAngle"] = q["BVAngle"]
        oP, oV = N.helical_to_fan(proj, z, **p)
    P, V = dd2.HelicalToFan_routine(proj, cfg, z)
    np.testing.assert_array_equal(P, oP)
    np.testing.assert_array_equal(V, oV)
    dev = torch.device("cuda", 0)
    d_raw = torch.from_numpy(proj).to(dev)
    n = z.size
    T, W = p["DefTimes"], p["DetWidth"]
    for layout in (0, 1):
        out = torch.full((n * T * W,), float("nan"), device=dev)
        views = torch.full((n * T,), float("nan"), device=dev)
        s = torch.cuda.current_stream(dev)
        call("ddfan_helical_to_fan_dev", ctypes.c_void_p(d_raw.data_ptr()), proj.shape[0],
             z.ctypes.data_as(ctypes.c_void_p), n, p["SD"], p["SO"], p["BVAngle"], W, p["DetHeight"],
             p["PerDetW"], p["PerDetH"], T, p["DetCenterW"], p["SpiralPitchFactor"], layout,
             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(views.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        torch.cuda.synchronize(dev)
        if layout == 0:
            got_P = out.cpu().numpy().reshape(n, T, W).transpose(1, 2, 0)
            got_V = views.cpu().numpy().reshape(n, T).T
        else:
            got_P = out.cpu().numpy().reshape(T, W, n)
            got_V = views.cpu().numpy().reshape(T, n)
        np.testing.assert_array_equal(got_P, oP)
        np.testing.assert_array_equal(got_V, oV)


@pytest.mark.gpu
def test_gpu_rebin_full_detector_size():
    """A Siemens-sized detector (736 channels x 64 rows, 2304 views per
    rotation) over 48 slices: every slice bit-identical to the restatement on
    a sample of slices, and all outputs finite."""
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    proj, z, p = synthetic(W=736, H=64, T=2304, rot=3.2, PW=1.2858, PH=1.0947, CW=369.625, pitch=0.8,
                           SLN=48, seed=7, edges=False)
    P, V = dd2.HelicalToFanFunc_mex(proj, z, z.size, **p)
    assert np.isfinite(P).all() and np.isfinite(V).all()
    for s in (0, 17, 47):
        oP, oV = N.helical_to_fan(proj, z[s:s + 1], **p)
        np.testing.assert_array_equal(P[s], oP[:, :, 0])
        np.testing.assert_array_equal(V[s], oV[:, 0])
