"""DICOM-CT-PD projection input: the byte converters pinned to the reference's
own cov_*.cpp, the header and pixel reading on files written here (the AAPM
data are not available), and the device conversion feeding the rebinning."""
import ctypes
import os
import struct

import numpy as np
import pytest

from aapm_lowdosectimagerecon_competition_b200 import ctpd

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
COVLIB = os.path.join(ROOT, "oracle", "_ref", "libref_cov.so")

EXPLICIT, IMPLICIT = "1.2.840.10008.1.2.1", "1.2.840.10008.1.2"


# ---------------------------------------------------------------- a minimal writer (tests only)

def _pad(b):
    return b if len(b) % 2 == 0 else b + b" "


def _element(g, e, vr, val, explicit):
    val = _pad(val) if vr not in (b"OB", b"OW", b"UN") else (val if len(val) % 2 == 0 else val + b"\x00")
    if explicit or g == 0x0002:
        if vr in (b"OB", b"OW", b"UN", b"SQ", b"UT"):
            return struct.pack("<HH2sHI", g, e, vr, 0, len(val)) + val
        return struct.pack("<HH2sH", g, e, vr, len(val)) + val
    return struct.pack("<HHI", g, e, len(val)) + val


def write_dicom(path, elements, ts=EXPLICIT):
    """elements: list of ((g, e), vr, bytes), written in tag order."""
    meta = _element(0x0002, 0x0010, b"UI", ts.encode() + b"\x00" * (len(ts) % 2), True)
    meta = _element(0x0002, 0x0000, b"UL", struct.pack("<I", len(meta)), True) + meta
    body = b"".join(_element(g, e, vr, v, ts == EXPLICIT) for (g, e), vr, v in sorted(elements))
    with open(path, "wb") as f:
        f.write(b"\x00" * 128 + b"DICM" + meta + body)


GEOM = dict(HU=0.0192, DCD=500.0, pitch=0.6, rows=16, cols=40, tsp=1.2858, asp=1.0947, ang=1.25, axial=-120.5,
            radial=595.0, cx=20.25, cy=8.5, sdd=1085.6, dphi=0.001, dz=3.3613e-4, drho=0.0, steps=48)


def projection_elements(pix, geo=GEOM, seq_first=False):
    f4 = lambda v: struct.pack("<f", v)
    el = [((0x0018, 0x0061), b"UN", b"%.4f " % geo["HU"]),
          ((0x0018, 0x0090), b"UN", b"%.1f" % geo["DCD"]),
          ((0x0018, 0x9311), b"UN", struct.pack("<d", geo["pitch"])),
          ((0x0028, 0x0010), b"US", struct.pack("<H", pix.shape[0])),
          ((0x0028, 0x0011), b"US", struct.pack("<H", pix.shape[1])),
          ((0x0028, 0x0100), b"US", struct.pack("<H", 16)),
          ((0x0028, 0x0103), b"US", struct.pack("<H", 0)),
          ((0x7029, 0x1002), b"UN", f4(geo["tsp"])),
          ((0x7029, 0x1006), b"UN", f4(geo["asp"])),
          ((0x7029, 0x100B), b"UN", b"CYLINDRICAL "),
          ((0x7029, 0x1010), b"UN", struct.pack("<H", geo["rows"])),
          ((0x7029, 0x1011), b"UN", struct.pack("<H", geo["cols"])),
          ((0x7031, 0x1001), b"UN", f4(geo["ang"])),
          ((0x7031, 0x1002), b"UN", f4(geo["axial"])),
          ((0x7031, 0x1003), b"UN", f4(geo["radial"])),
          ((0x7031, 0x1031), b"UN", f4(geo["sdd"])),
          ((0x7031, 0x1033), b"UN", f4(geo["cx"]) + f4(geo["cy"])),
          ((0x7033, 0x100B), b"UN", f4(geo["dphi"])),
          ((0x7033, 0x100C), b"UN", f4(geo["dz"])),
          ((0x7033, 0x100D), b"UN", f4(geo["drho"])),
          ((0x7033, 0x1013), b"UN", struct.pack("<H", geo["steps"])),
          ((0x7033, 0x1065), b"UN", np.linspace(1e5, 2e5, geo["cols"]).astype("<f4").tobytes()),
          ((0x7FE0, 0x0010), b"OW", pix.astype("<u2").tobytes())]
    return el


def write_scan(folder, views, ts=EXPLICIT):
    """views: uint16 (n, cols, rows) stored pixels, written as files 0001.dcm ..."""
    os.makedirs(folder, exist_ok=True)
    for i, v in enumerate(views):
        write_dicom(os.path.join(folder, "%04d.dcm" % (i + 1)), projection_elements(v), ts)


# ---------------------------------------------------------------- CPU

@pytest.mark.skipif(not os.path.exists(COVLIB), reason="reference converters not compiled (make -C oracle ref)")
def test_byte_converters_match_the_reference():
    L = ctypes.CDLL(COVLIB)
    P, D = ctypes.c_char_p, ctypes.c_double
    L.ddref_cov_4uint8_to_float.restype = D
    L.ddref_cov_4uint8_to_float.argtypes = [P]
    L.ddref_cov_8uint8_to_double.restype = D
    L.ddref_cov_8uint8_to_double.argtypes = [P]
    L.ddref_cov_uint8_to_double.restype = D
    L.ddref_cov_uint8_to_double.argtypes = [P]
    L.ddref_cov_8uint8_to_2floats.argtypes = [P, ctypes.POINTER(D), ctypes.POINTER(D)]
    L.ddref_cov_uint8_to_PhoStat.argtypes = [P, ctypes.c_int, ctypes.c_void_p]
    rng = np.random.default_rng(0)
    for _ in range(200):
        b = rng.integers(0, 256, 8, dtype=np.uint8).tobytes()
        r = L.ddref_cov_4uint8_to_float(b)
        o = ctpd.cov_4uint8_to_float(b)
        assert (np.isnan(r) and np.isnan(o)) or r == o
        r = L.ddref_cov_8uint8_to_double(b)
        o = ctpd.cov_8uint8_to_double(b)
        assert (np.isnan(r) and np.isnan(o)) or r == o
        x, y = D(), D()
        L.ddref_cov_8uint8_to_2floats(b, ctypes.byref(x), ctypes.byref(y))
        ox, oy = ctpd.cov_8uint8_to_2floats(b)
        assert (np.isnan(x.value) and np.isnan(ox)) or x.value == ox
        assert (np.isnan(y.value) and np.isnan(oy)) or y.value == oy
    for s in (b"0.0192 ", b"500", b"-1.5e-3 ", b" 42.25", b"7.", b"1e3x", b"abc", b"+3.5 "):
        assert L.ddref_cov_uint8_to_double(s) == ctpd.cov_uint8_to_double(s), s
    pho = np.linspace(1, 2, 37).astype("<f4").tobytes()
    out = np.zeros(37)
    L.ddref_cov_uint8_to_PhoStat(pho, 37, out.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_array_equal(out, ctpd.cov_uint8_to_PhoStat(pho, 37))


@pytest.mark.parametrize("ts", [EXPLICIT, IMPLICIT])
def test_collect_recon_cfg_reads_the_geometry_tags(tmp_path, ts):
    pix = np.arange(40 * 16, dtype=np.uint16).reshape(40, 16)
    f = str(tmp_path / "a.dcm")
    write_dicom(f, projection_elements(pix), ts)
    cfg = ctpd.CollectReconCfg(f)
    f32 = lambda v: float(np.float32(v))
    g = GEOM
    assert cfg["HUCalibrationFactor"] == 0.0192 and cfg["DataCollectionDiameter"] == 500.0
    assert cfg["SpiralPitchFactor"] == 0.6
    assert cfg["NumberofDetectorRows"] == 16 and cfg["NumberofDetectorColumns"] == 40
    assert cfg["DetectorElementTransverseSpacing"] == f32(g["tsp"])
    assert cfg["DetectorElementAxialSpacing"] == f32(g["asp"])
    assert cfg["DetectorFocalCenterAngularPosition"] == f32(g["ang"])
    assert cfg["DetectorFocalCenterRadialDistance"] == f32(g["radial"])
    assert cfg["ConstantRadialDistance"] == f32(g["sdd"])
    assert cfg["DetectorCentralElement"] == {"X": f32(g["cx"]), "Y": f32(g["cy"])}
    assert cfg["NumberofSourceAngularSteps"] == 48 and cfg["SpiralPitchGE"] == 0.6 * 16
    assert cfg["PhotonStatistics"].shape == (40,) and cfg["DetectorType"].startswith("CYLINDRICAL")
    np.testing.assert_array_equal(ctpd.pixels(f), pix)


def test_read_proj_layout_and_view_order(tmp_path):
    rng = np.random.default_rng(1)
    views = rng.integers(0, 4096, (6, 40, 16), dtype=np.uint16)
    write_scan(str(tmp_path / "scan"), views)
    proj, cfg = ctpd.readProj(str(tmp_path / "scan"))
    assert cfg["NumOfDataViews"] == 6
    # (views, DetWidth, DetHeight) = MATLAB (DetHeight, DetWidth, views) after permute, views reversed
    assert proj.dtype == np.float32 and proj.shape == (6, 40, 16)
    np.testing.assert_array_equal(proj, views[::-1].astype(np.float32))


def test_image_cfg_and_recon_conf(tmp_path):
    f = str(tmp_path / "img.dcm")
    el = [((0x0018, 0x0050), b"DS", b"1.0 "), ((0x0018, 0x1100), b"DS", b"380.0 "),
          ((0x0028, 0x0010), b"US", struct.pack("<H", 512)), ((0x0028, 0x0011), b"US", struct.pack("<H", 512)),
          ((0x0028, 0x0030), b"DS", b"0.742\\0.742 "), ((0x0028, 0x1052), b"DS", b"-1024 "),
          ((0x0028, 0x1053), b"DS", b"1 ")]
    write_dicom(f, el)
    img = ctpd.CollectImageCfg(f)
    assert img["Width"] == 512 and img["Height"] == 512 and img["PixelSize"] == 380.0 / 512
    assert img["PixelSpacing"] == [0.742, 0.742] and img["RescaleIntercept"] == -1024.0
    pf = str(tmp_path / "p.dcm")
    write_dicom(pf, projection_elements(np.zeros((40, 16), np.uint16)))
    conf = ctpd.ConvertToReconConf(ctpd.CollectReconCfg(pf), img, 64)
    assert conf["recon"] == {"XN": 512, "YN": 512, "dx": 380.0 / 512} and conf["SLN"] == 64
    assert conf["acq"]["DNU"] == 40 and conf["acq"]["PN"] == 48
    assert conf["acq"]["sid"] == float(np.float32(595.0)) and conf["acq"]["detCntIdx"] == 20.25


def test_unsupported_files_are_errors(tmp_path):
    f = str(tmp_path / "x.dcm")
    with open(f, "wb") as fh:
        fh.write(b"not dicom")
    with pytest.raises(ctpd.DicomError):
        ctpd.read_dataset(f)
    write_dicom(f, projection_elements(np.zeros((40, 16), np.uint16)), ts="1.2.840.10008.1.2.4.50")
    with pytest.raises(ctpd.DicomError):
        ctpd.read_dataset(f)


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_device_conversion_equals_host_read_and_feeds_rebinning(tmp_path):
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    from oracle import np_oracle as N
    rng = np.random.default_rng(2)
    n = 4 * GEOM["steps"]
    views = rng.integers(0, 60000, (n, 40, 16), dtype=np.uint16)
    folder = str(tmp_path / "scan")
    write_scan(folder, views)
    proj, cfg = ctpd.readProj(folder)
    d_proj, cfg2 = ctpd.readProj_device(folder)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_proj.cpu().numpy(), proj)
    assert cfg2["NumOfDataViews"] == cfg["NumOfDataViews"]
    # DICOM -> rebinning with the header's geometry, as reconscript.m:17-25
    p = dd2.rebin_params(dict(cfg, DetectorFocalCenterAngularPosition=cfg["DetectorFocalCenterAngularPosition"]))
    f = np.float32
    h = p["SpiralPitchFactor"] * p["PerDetH"] * f(p["DetHeight"]) * p["SO"] / p["SD"]
    dz = h / f(p["DefTimes"])
    z = np.linspace(float(h), float(dz) * n - float(h), 5).astype(np.float32)
    P, V = dd2.HelicalToFan_routine(proj, cfg, z)
    oP, oV = N.helical_to_fan(proj, z, **p)
    np.testing.assert_array_equal(P, oP)
    np.testing.assert_array_equal(V, oV)
