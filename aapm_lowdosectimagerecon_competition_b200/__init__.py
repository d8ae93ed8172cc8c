"""B200-native fan-beam multi-slice distance-driven projector, backprojector
and OS-SART/FISTA solver -- a drop-in for the MultiSlicesProjGPU /
MultiSlicesBackGPU / OSSART_AAPM path of the AAPM low-dose CT reconstruction
code.  All compute runs in the sm_100a kernels of libddfan.so.
"""
from ._lib import (BACK_ADJ, BACK_REF, SAT_FP32, SAT_FP64, SAT_HILO, DdfanError, LIB_PATH,
                   load as load_library)
from .dd2 import (DD2MutiSlices, MultiSlicesBackGPU, MultiSlicesProjGPU, OSSART_AAPM,
                  default_start_idx, fan_geometry)

__all__ = [
    "BACK_ADJ", "BACK_REF", "SAT_FP32", "SAT_FP64", "SAT_HILO", "DdfanError", "LIB_PATH",
    "load_library", "DD2MutiSlices", "MultiSlicesBackGPU", "MultiSlicesProjGPU", "OSSART_AAPM",
    "default_start_idx", "fan_geometry",
]
