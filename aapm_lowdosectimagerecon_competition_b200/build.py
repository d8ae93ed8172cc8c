"""Builds libddfan.so in-tree for sm_100a (nvcc; no CPU fallback exists).

    python -m aapm_lowdosectimagerecon_competition_b200.build
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libddfan.so")
SOURCES = ["ddfan.cu", "ddfan_solver.cu", "ddfan_ps.cu", "ddfan_noalloc.cu", "ddfan_rebin.cu", "ddfan_batch.cu"]
HEADERS = ["ddfan_device.cuh", "ddfan_kernels.cuh", "ddfan_proj_kernels.cuh", "ddfan_plan.h", "ddfan_ps.h",
           "ddfan_ps_kernels.cuh", "ddfan_dd_kernels.cuh", "ddfan_solver.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "ddfan.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile every CUDA source of the package into libddfan.so."""
    if not force and not _stale():
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        cmd = ["nvcc", *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
               "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run(["nvcc", *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
