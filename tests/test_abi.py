"""The C ABI library: it loads, exports every entry point of include/ddfan.h,
and fails loudly (status + message, never a CPU fallback) without a GPU.
CPU only: no kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

import aapm_lowdosectimagerecon_competition_b200 as pkg
from aapm_lowdosectimagerecon_competition_b200 import _lib, configs, dd2
from oracle import np_oracle as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ddfan.h")).read()
    return sorted(set(re.findall(r"DDFAN_API\s+[\w\s\*]+?\b(ddfan_\w+)\s*\(", src)))


def test_header_declares_the_mex_and_solver_entry_points():
    names = header_functions()
    for must in ("ddfan_MultiSlicesProjGPU", "ddfan_MultiSlicesBackGPU", "ddfan_OSSART_AAPM",
                 "ddfan_plan_create", "ddfan_proj_dev", "ddfan_back_dev", "ddfan_ossart_create",
                 "ddfan_ossart_iterate", "ddfan_last_error", "ddfan_fan_geometry"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert set(header_functions()) <= set(_lib.SIGNATURES)


def test_python_signatures_match_header_arity():
    src = open(os.path.join(ROOT, "include", "ddfan.h")).read()
    for name, (res, args) in _lib.SIGNATURES.items():
        m = re.search(r"DDFAN_API[^;(]*\b%s\s*\(([^;]*)\)\s*;" % name, src, re.S)
        assert m, name
        params = m.group(1).strip()
        n = 0 if params in ("", "void") else len(re.sub(r"/\*.*?\*/", "", params, flags=re.S).split(","))
        assert n == len(args), (name, n, len(args))


def test_fan_geometry_matches_matlab_restatement():
    for sid, sdd, DNU, w, cnt in [(595.0, 1085.6, 736, 1.2858, 368.5), (541.0, 949.0, 888, 1.0239, 444.5),
                                  (595.0, 1085.6, 736, 1.2858, 368.75)]:
        x0, y0, xds, yds = dd2.fan_geometry(np.float32(sid), np.float32(sdd), DNU, np.float32(w),
                                            np.float32(cnt))
        a0, b0, axs, ays = N.fan_geometry(sid, sdd, DNU, w, cnt)
        assert x0 == a0 and y0 == b0
        # single-precision sin/cos of different libraries: a few ulp
        np.testing.assert_allclose(xds, axs, rtol=1e-6, atol=2e-4)
        np.testing.assert_allclose(yds, ays, rtol=1e-6, atol=2e-4)


def test_bad_arguments_return_status_not_exit():
    lib = _lib.load()
    rc = lib.ddfan_fan_geometry(595.0, 1085.6, 0, 1.0, 1.0, None, None, None, None)
    assert rc == 1 and b"bad arguments" in lib.ddfan_last_error()


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly():
    s = configs.scaled(configs.c2(SLN=2), XN=16, DNU=24, PN=8)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    with pytest.raises(pkg.DdfanError) as e:
        dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN,
                               np.ones((s.YN, s.XN, s.SLN), np.float32), s.dx)
    assert "CUDA" in str(e.value) or "device" in str(e.value)


@pytest.mark.parametrize("XN,YN,DNU,code", [(1025, 64, 64, 4), (64, 1025, 64, 4), (64, 64, 1024, 4),
                                            (1024, 1024, 1023, None)])
def test_line_length_limit_is_checked_before_device_work(XN, YN, DNU, code):
    """Image lines and detector rows of up to 1024 cells; longer ones return
    DDFAN_ERR_UNSUPPORTED from plan creation and the no-alloc projection,
    before any device is touched (so the same on a machine without one)."""
    lib = _lib.load()
    x0, y0, xds, yds = dd2.fan_geometry(np.float32(595.0), np.float32(1085.6), DNU, np.float32(1.2858),
                                        np.float32((DNU + 1) / 2.0))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    h = ctypes.c_void_p()
    rc = lib.ddfan_plan_create(ctypes.byref(h), x0, y0, DNU, P(xds), P(yds), (DNU + 1) / 2.0, 0.0, 0.0, XN, YN,
                               0.7, None, 8, 96, 1, 0)
    if h.value:
        lib.ddfan_plan_destroy(h)
    dummy = np.zeros(4, np.float32)
    rc2 = lib.ddfan_proj_noalloc(x0, y0, DNU, P(xds), P(yds), 0.0, 0.0, P(dummy), 96, XN, YN, 8, P(dummy), 0.7,
                                 None, 1, P(dummy), None)
    if code is None:  # at the limit: passes the size check (then needs a device)
        assert rc != 4 and rc2 != 4
        if not torch.cuda.is_available():
            assert rc == 2 and rc2 == 2
    else:
        assert rc == code and rc2 == code
        assert b"1024" in lib.ddfan_last_error()


def test_argument_validation_before_any_device_work():
    s = configs.scaled(configs.c2(SLN=2), XN=16, DNU=24, PN=8)
    x0, y0, xds, yds = dd2.fan_geometry(s.sid, s.sdd, s.DNU, s.detCellWidth, s.detCntIdx)
    with pytest.raises(ValueError):
        dd2.MultiSlicesProjGPU(x0, y0, s.DNU, xds, yds, 0, 0, s.hangs(), s.PN, s.XN, s.YN, s.SLN,
                               np.ones((3, 3, 3), np.float32), s.dx)
    with pytest.raises(ValueError):
        dd2.MultiSlicesBackGPU(x0, y0, s.DNU, xds, yds, s.detCntIdx, 0, 0, s.hangs(), s.PN, s.XN, s.YN,
                               s.SLN, np.ones((s.PN, s.DNU, s.SLN), np.float32), s.dx, back="bogus")


def test_default_start_idx_is_the_matlab_formula():
    # ceil((ii - 1) / numgpu * SLN), ii = 1..numgpu (AAPM_script/DD2MutiSlices.m:95-101)
    for SLN, n in [(512, 3), (512, 4), (7, 2), (128, 8)]:
        exp = [int(np.ceil((ii - 1) / n * SLN)) for ii in range(1, n + 1)]
        assert list(dd2.default_start_idx(SLN, n)) == exp
