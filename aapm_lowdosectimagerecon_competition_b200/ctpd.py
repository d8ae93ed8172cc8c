"""DICOM-CT-PD projection input: the on-disk format of the AAPM low-dose CT
challenge data, read the way the reference reads it.

Reference routines mirrored (paths relative to the reference project root):
  readProj            AAPM_script/readProj.m:31-56
  CollectReconCfg     AAPM_script/CollectReconCfg.m:2-95
  CollectImageCfg     AAPM_script/CollectImageCfg.m:1-31
  ConvertToReconConf  AAPM_script/ConvertToReconConf.m:21-33
  cov_*               AAPM_script/cov_uint8_to_double.cpp, cov_8uint8_to_double.cpp,
                      cov_4uint8_to_float.cpp, cov_8uint8_to_2floats.cpp,
                      cov_uint8_to_PhoStat.cpp

The DICOM reader is this project's own minimal Part-10 parser: little-endian
explicit or implicit VR, uncompressed pixel data, defined-length elements
(sequences of undefined length are skipped).  The reference uses MATLAB's
dicominfo with a private dictionary; it reads the private geometry tags as raw
bytes and re-interprets them with the cov_* helpers, which are restated here.
Pixel values are the stored integers, not rescaled (readProj.m:46).
"""
import glob
import os
import struct

import numpy as np

# VRs whose explicit-VR header has a 2-byte reserved field and a 4-byte length
_LONG_VR = {b"OB", b"OD", b"OF", b"OL", b"OW", b"SQ", b"UC", b"UN", b"UR", b"UT", b"OV", b"SV", b"UV"}
PIXEL_DATA = (0x7FE0, 0x0010)


class DicomError(ValueError):
    pass


def read_dataset(path, stop_before_pixels=False):
    """Elements of a DICOM Part-10 file: {(group, element): raw value bytes}."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 132 or data[128:132] != b"DICM":
        raise DicomError("%s: not a DICOM Part-10 file" % path)
    pos, out = 132, {}
    ts = None
    explicit = True
    while pos + 8 <= len(data):
        g, e = struct.unpack_from("<HH", data, pos)
        # the file meta group is explicit VR; the data set follows the transfer syntax
        exp = True if g == 0x0002 else explicit
        if g == 0xFFFE:  # item / delimiters at top level: skip their header
            pos += 8
            continue
        if exp:
            vr = data[pos + 4:pos + 6]
            if vr in _LONG_VR:
                (ln,) = struct.unpack_from("<I", data, pos + 8)
                hdr = 12
            else:
                (ln,) = struct.unpack_from("<H", data, pos + 6)
                hdr = 8
        else:
            (ln,) = struct.unpack_from("<I", data, pos + 4)
            hdr = 8
        pos += hdr
        if ln == 0xFFFFFFFF:
            if (g, e) == PIXEL_DATA:
                raise DicomError("%s: encapsulated (compressed) pixel data is not supported" % path)
            pos = _skip_undefined(data, pos)
            continue
        if (g, e) == PIXEL_DATA and stop_before_pixels:
            break
        out[(g, e)] = data[pos:pos + ln]
        pos += ln
        if (g, e) == (0x0002, 0x0010):
            ts = out[(g, e)].rstrip(b"\x00 ").decode("ascii", "replace")
            if ts == "1.2.840.10008.1.2":
                explicit = False
            elif ts in ("1.2.840.10008.1.2.1",):
                explicit = True
            else:
                raise DicomError("%s: transfer syntax %s is not supported (little-endian, uncompressed only)"
                                 % (path, ts))
    return out


def _skip_undefined(data, pos):
    """Past the sequence delimiter of an undefined-length element."""
    depth = 1
    while pos + 8 <= len(data):
        g, e = struct.unpack_from("<HH", data, pos)
        (ln,) = struct.unpack_from("<I", data, pos + 4)
        pos += 8
        if g == 0xFFFE and e == 0xE0DD:  # sequence delimitation
            depth -= 1
            if depth == 0:
                return pos
        elif g == 0xFFFE and e == 0xE000:  # item
            if ln != 0xFFFFFFFF:
                pos += ln
        elif g == 0xFFFE and e == 0xE00D:  # item delimitation
            pass
        else:
            raise DicomError("undefined-length sequences with nested elements are not supported")
    raise DicomError("unterminated sequence")


# ---------------------------------------------------------------- cov_* helpers

def cov_uint8_to_double(b):
    """atof of the bytes (a decimal string), cov_uint8_to_double.cpp:17-22."""
    s = bytes(b).split(b"\x00", 1)[0].decode("ascii", "replace").strip()
    num = ""
    for ch in s:  # atof: the longest leading number
        if ch in "+-0123456789.eE" and not (ch in "+-" and num and num[-1] not in "eE"):
            num += ch
        else:
            break
    while num:
        try:
            return float(num)
        except ValueError:
            num = num[:-1]
    return 0.0


def cov_8uint8_to_double(b):
    """Little-endian float64 from 8 bytes, cov_8uint8_to_double.cpp:17-30."""
    return struct.unpack("<d", bytes(b[:8]))[0]


def cov_4uint8_to_float(b):
    """Little-endian float32 from 4 bytes, as a double (cov_4uint8_to_float.cpp:17-27)."""
    return float(struct.unpack("<f", bytes(b[:4]))[0])


def cov_8uint8_to_2floats(b):
    """Two little-endian float32 from 8 bytes (cov_8uint8_to_2floats.cpp:17-35)."""
    x, y = struct.unpack("<ff", bytes(b[:8]))
    return float(x), float(y)


def cov_uint8_to_PhoStat(b, n):
    """n little-endian float32, as doubles (cov_uint8_to_PhoStat.cpp:22-38)."""
    return np.frombuffer(bytes(b[:4 * int(n)]), dtype="<f4").astype(np.float64)


def _u16(b):
    """double(b(2)) * 2^8 + double(b(1)) (CollectReconCfg.m:21-26)."""
    return float(b[1]) * 256.0 + float(b[0])


# ---------------------------------------------------------------- headers

def CollectReconCfg(FileName, dictionaryFile=None):
    """Scan geometry from one projection file's tags (CollectReconCfg.m:2-95).
    The private tags are read as raw bytes; dictionaryFile is accepted for the
    reference's signature and not needed."""
    d = read_dataset(FileName, stop_before_pixels=True)

    def tag(g, e):
        try:
            return d[(g, e)]
        except KeyError:
            raise DicomError("%s: tag (%04X,%04X) missing" % (FileName, g, e))

    cfg = {}
    cfg["HUCalibrationFactor"] = cov_uint8_to_double(tag(0x0018, 0x0061))
    cfg["DataCollectionDiameter"] = cov_uint8_to_double(tag(0x0018, 0x0090))
    cfg["SpiralPitchFactor"] = cov_8uint8_to_double(tag(0x0018, 0x9311))
    cfg["NumberofDetectorRows"] = _u16(tag(0x7029, 0x1010))
    cfg["NumberofDetectorColumns"] = _u16(tag(0x7029, 0x1011))
    cfg["DetectorElementTransverseSpacing"] = cov_4uint8_to_float(tag(0x7029, 0x1002))
    cfg["DetectorElementAxialSpacing"] = cov_4uint8_to_float(tag(0x7029, 0x1006))
    cfg["DetectorType"] = bytes(tag(0x7029, 0x100B)).decode("latin-1")
    cfg["DetectorFocalCenterAngularPosition"] = cov_4uint8_to_float(tag(0x7031, 0x1001))
    cfg["DetectorFocalCenterAxialPosition"] = cov_4uint8_to_float(tag(0x7031, 0x1002))
    cfg["DetectorFocalCenterRadialDistance"] = cov_4uint8_to_float(tag(0x7031, 0x1003))
    x, y = cov_8uint8_to_2floats(tag(0x7031, 0x1033))
    cfg["DetectorCentralElement"] = {"X": x, "Y": y}
    cfg["ConstantRadialDistance"] = cov_4uint8_to_float(tag(0x7031, 0x1031))
    cfg["SourceAngularPositionShift"] = cov_4uint8_to_float(tag(0x7033, 0x100B))
    cfg["SourceAxialPositionShift"] = cov_4uint8_to_float(tag(0x7033, 0x100C))
    cfg["SourceRadialDistanceShift"] = cov_4uint8_to_float(tag(0x7033, 0x100D))
    cfg["NumberofSourceAngularSteps"] = _u16(tag(0x7033, 0x1013))
    cfg["PhotonStatistics"] = cov_uint8_to_PhoStat(tag(0x7033, 0x1065), int(cfg["NumberofDetectorColumns"]))
    cfg["SpiralPitchGE"] = cfg["SpiralPitchFactor"] * cfg["NumberofDetectorRows"]
    return cfg


def _ds(b):
    vals = [v for v in bytes(b).decode("ascii", "replace").strip("\x00 ").split("\\") if v.strip()]
    out = [float(v) for v in vals]
    return out[0] if len(out) == 1 else out


def _us(b):
    return struct.unpack("<H", bytes(b[:2]))[0]


def _fd(b):
    vals = struct.unpack("<%dd" % (len(b) // 8), bytes(b[:8 * (len(b) // 8)]))
    return vals[0] if len(vals) == 1 else list(vals)


def CollectImageCfg(FileName):
    """Reconstruction grid and display fields of a reconstructed-image file
    (CollectImageCfg.m:1-31); Width/Height are Columns/Rows as dicominfo names them."""
    d = read_dataset(FileName, stop_before_pixels=True)
    g = lambda t, f, default=None: f(d[t]) if t in d else default
    cfg = {"Width": g((0x0028, 0x0011), _us), "Height": g((0x0028, 0x0010), _us),
           "BitDepth": g((0x0028, 0x0101), _us), "SliceThickness": g((0x0018, 0x0050), _ds),
           "KVP": g((0x0018, 0x0060), _ds), "DataCollectionDiameter": g((0x0018, 0x0090), _ds),
           "ReconstructionDiameter": g((0x0018, 0x1100), _ds),
           "SingleCollimationWidth": g((0x0018, 0x9306), _fd), "TotalCollimationWidth": g((0x0018, 0x9307), _fd),
           "TableSpeed": g((0x0018, 0x9309), _fd), "TableFeedPerRotation": g((0x0018, 0x9310), _fd),
           "SpiralPitchFactor": g((0x0018, 0x9311), _fd),
           "DataCollectionCenterPatient": g((0x0018, 0x9313), _fd),
           "ReconstructionTargetCenterPatient": g((0x0018, 0x9318), _fd),
           "Rows": g((0x0028, 0x0010), _us), "Columns": g((0x0028, 0x0011), _us),
           "PixelSpacing": g((0x0028, 0x0030), _ds), "WindowCenter": g((0x0028, 0x1050), _ds),
           "WindowWidth": g((0x0028, 0x1051), _ds), "RescaleIntercept": g((0x0028, 0x1052), _ds),
           "RescaleSlope": g((0x0028, 0x1053), _ds)}
    if cfg["ReconstructionDiameter"] is not None and cfg["Width"]:
        cfg["PixelSize"] = cfg["ReconstructionDiameter"] / cfg["Width"]
    return cfg


def ConvertToReconConf(cfg, cfgRecon, SLN):
    """The conf struct the projector and OSSART_AAPM take (ConvertToReconConf.m:21-33)."""
    return {"recon": {"XN": int(cfgRecon["Width"]), "YN": int(cfgRecon["Height"]), "dx": cfgRecon["PixelSize"]},
            "SLN": int(SLN),
            "acq": {"sid": cfg["DetectorFocalCenterRadialDistance"], "DNU": int(cfg["NumberofDetectorColumns"]),
                    "PN": int(cfg["NumberofSourceAngularSteps"]), "sdd": cfg["ConstantRadialDistance"],
                    "detCellWidth": cfg["DetectorElementTransverseSpacing"],
                    "detCntIdx": cfg["DetectorCentralElement"]["X"]}}


# ---------------------------------------------------------------- projections

def pixels(FileName, d=None):
    """Stored pixel values of one file as a (Rows, Columns) array (no rescale)."""
    d = read_dataset(FileName) if d is None else d
    rows, cols = _us(d[(0x0028, 0x0010)]), _us(d[(0x0028, 0x0011)])
    bits = _us(d[(0x0028, 0x0100)])
    signed = _us(d.get((0x0028, 0x0103), b"\x00\x00")) == 1
    dt = {8: "i1" if signed else "u1", 16: "<i2" if signed else "<u2", 32: "<i4" if signed else "<u4"}.get(bits)
    if dt is None:
        raise DicomError("%s: %d bits allocated is not supported" % (FileName, bits))
    raw = d[PIXEL_DATA]
    return np.frombuffer(raw, dtype=dt, count=rows * cols).reshape(rows, cols)


def projection_files(FilePath):
    """The *.dcm files of a projection folder in the order MATLAB's dir lists them (by name)."""
    files = sorted(glob.glob(os.path.join(FilePath, "*.dcm")))
    if not files:
        raise DicomError("%s: no .dcm files" % FilePath)
    return files


def read_views(FilePath):
    """Stored pixels of every projection, stacked in file order: (views, Rows, Columns)."""
    files = projection_files(FilePath)
    first = pixels(files[0])
    out = np.empty((len(files),) + first.shape, dtype=first.dtype)
    out[0] = first
    for i, f in enumerate(files[1:], 1):
        p = pixels(f)
        if p.shape != first.shape:
            raise DicomError("%s: %s pixels, first file has %s" % (f, p.shape, first.shape))
        out[i] = p
    return out


def readProj(FilePath):
    """(proj, cfg) as readProj.m:31-56: proj float32 (TotalViews, DetWidth,
    DetHeight) -- MATLAB (DetHeight, DetWidth, TotalViews) after its permute --
    with the views in reverse file order (:54), cfg from the first file with
    NumOfDataViews."""
    files = projection_files(FilePath)
    dicts = glob.glob(os.path.join(FilePath, "*.txt"))
    cfg = CollectReconCfg(files[0], dicts[0] if dicts else None)
    cfg["NumOfDataViews"] = len(files)
    views = read_views(FilePath)
    W, H = int(cfg["NumberofDetectorColumns"]), int(cfg["NumberofDetectorRows"])
    if views.shape[1:] != (W, H):
        raise DicomError("projections are %s pixels, the header says %d columns x %d rows"
                         % (views.shape[1:], W, H))
    return np.ascontiguousarray(views[::-1].astype(np.float32)), cfg


def readProj_device(FilePath, device=None, stream=None):
    """readProj with the conversion on the GPU: the stored 16-bit pixels are
    uploaded (half the bytes of float32) and converted, views reversed, by
    ddfan_ctpd_views_to_raw into a float32 CUDA tensor (TotalViews, DetWidth,
    DetHeight) -- the input of ddfan_helical_to_fan_dev."""
    import ctypes

    import torch

    from ._lib import call
    files = projection_files(FilePath)
    cfg = CollectReconCfg(files[0])
    cfg["NumOfDataViews"] = len(files)
    views = read_views(FilePath)
    if views.dtype != np.uint16:
        raise DicomError("device conversion takes unsigned 16-bit pixels, got %s" % views.dtype)
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    st = torch.cuda.current_stream(dev) if stream is None else stream
    n, W, H = views.shape
    with torch.cuda.stream(st):
        src = torch.from_numpy(views.view(np.int16)).pin_memory().to(dev, non_blocking=True)
        out = torch.empty((n, W, H), dtype=torch.float32, device=dev)
    call("ddfan_ctpd_views_to_raw", ctypes.c_void_p(src.data_ptr()), n, W, H, 1, ctypes.c_void_p(out.data_ptr()),
         ctypes.c_void_p(st.cuda_stream))
    src.record_stream(st)
    return out, cfg
