"""ctypes binding of libddfan.so (the C ABI declared in include/ddfan.h).

The library is the only compute path: if it is missing or cannot be loaded,
every entry point raises -- there is no CPU fallback.
"""
import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libddfan.so")

OK = 0
SAT_FP32, SAT_HILO, SAT_FP64, SAT_DIRECT = 0, 1, 2, 3
BACK_REF, BACK_ADJ = 0, 1
SAT_MODES = {"fp32": SAT_FP32, "hilo": SAT_HILO, "fp64": SAT_FP64, "direct": SAT_DIRECT}
BACK_MODES = {"ref": BACK_REF, "adj": BACK_ADJ}

_f = ctypes.c_float
_i = ctypes.c_int
_p = ctypes.c_void_p
_sz = ctypes.c_size_t
_ll = ctypes.c_longlong

# name -> (restype, argtypes); mirrors include/ddfan.h
SIGNATURES = {
    "ddfan_last_error": (ctypes.c_char_p, []),
    "ddfan_version": (_i, []),
    "ddfan_tune_set_zl": (_i, [_i, _i]),
    "ddfan_tune_get_zl": (_i, [_i]),
    "ddfan_tune_set_nz": (_i, [_i, _i]),
    "ddfan_tune_get_nz": (_i, [_i]),
    "ddfan_plan_estimate_bytes": (_sz, [_i, _i, _i, _i, _i, _i]),
    "ddfan_ossart_estimate_bytes": (_sz, [_i, _i, _i, _i, _i, _i, _i]),
    "ddfan_fan_geometry": (_i, [_f, _f, _i, _f, _f, _p, _p, _p, _p]),
    "ddfan_MultiSlicesProjGPU": (_i, [_f, _f, _i, _p, _p, _f, _f, _p, _i, _i, _i, _i, _p, _f, _p, _p,
                                      _i, _i, _p]),
    "ddfan_MultiSlicesBackGPU": (_i, [_f, _f, _i, _p, _p, _f, _f, _f, _p, _i, _i, _i, _i, _p, _f, _p,
                                      _p, _i, _i, _i, _p]),
    "ddfan_plan_create": (_i, [_p, _f, _f, _i, _p, _p, _f, _f, _f, _i, _i, _f, _p, _i, _i, _i, _i]),
    "ddfan_plan_destroy": (None, [_p]),
    "ddfan_plan_device_bytes": (_sz, [_p]),
    "ddfan_cached_bytes": (_sz, [_i]),
    "ddfan_release_cached": (_i, [_i]),
    "ddfan_proj_dev": (_i, [_p, _p, _i, _i, _p, _p, _p]),
    "ddfan_back_dev": (_i, [_p, _p, _i, _i, _p, _p, _i, _p]),
    "ddfan_proj_noalloc": (_i, [_f, _f, _i, _p, _p, _f, _f, _p, _i, _i, _i, _i, _p, _f, _p, _i, _p, _p]),
    "ddfan_ossart_create": (_i, [_p, _f, _f, _i, _p, _p, _f, _f, _f, _p, _i, _i, _i, _i, _f, _p, _i,
                                 _i, _i, _i, _i, _i]),
    "ddfan_ossart_destroy": (None, [_p]),
    "ddfan_ossart_device_bytes": (_sz, [_p]),
    "ddfan_ossart_set_sinogram": (_i, [_p, _p, _i, _p]),
    "ddfan_ossart_set_image": (_i, [_p, _p, _i, _p]),
    "ddfan_ossart_iterate": (_i, [_p, _i, _i, _p]),
    "ddfan_ossart_get_image": (_i, [_p, _p, _i, _p]),
    "ddfan_ossart_image_ptr": (_p, [_p]),
    "ddfan_ossart_launches_per_iter": (_i, [_p]),
    "ddfan_ossart_profile": (_i, [_p, _i, _p, _p, _p]),
    "ddfan_batch_create": (_i, [_p, _p, _i]),
    "ddfan_batch_destroy": (None, [_p]),
    "ddfan_batch_iterate": (_i, [_p, _i, _i, _p]),
    "ddfan_batch_launches_per_iter": (_i, [_p]),
    "ddfan_OSSART_AAPM": (_i, [_f, _f, _i, _p, _p, _f, _f, _f, _p, _p, _i, _i, _i, _i, _f, _p, _p, _i,
                               _i, _i, _i, _i, _i, _p]),
    "ddfan_HelicalToFan": (_i, [_p, _p, _p, _ll, _p, _i, _f, _f, _f, _i, _i, _f, _f, _i, _f, _f]),
    "ddfan_helical_to_fan_dev": (_i, [_p, _ll, _p, _i, _f, _f, _f, _i, _i, _f, _f, _i, _f, _f, _i, _p, _p,
                                      _p]),
    "ddfan_ctpd_views_to_raw": (_i, [_p, _ll, _i, _i, _i, _p, _p]),
}

_LIB = None


class DdfanError(RuntimeError):
    """A libddfan entry point returned a non-zero status."""

    def __init__(self, fn, code, msg):
        super().__init__("%s failed (status %d): %s" % (fn, code, msg))
        self.code = code


def load():
    """Load libddfan.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libddfan.so not built (%s); run "
                              "`python -m aapm_lowdosectimagerecon_competition_b200.build`" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def call(name, *args):
    """Call an int-returning entry point; raise DdfanError on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        msg = lib.ddfan_last_error()
        raise DdfanError(name, rc, msg.decode() if msg else "")
    return rc
