// Test-infrastructure harness around the reference's own per-GPU host drivers.
//
// The reference sources (AAPM_script/MultiSlicesProjGPU.cu and
// AAPM_script/MultiSlicesBackGPU.cu) are compiled unmodified next to this file
// (see oracle/Makefile); this harness only gives their per-GPU drivers a C
// entry point so tests can call them through ctypes:
//   DD2::DD2_gpu_proj_branchless_sat2d  (AAPM_script/MultiSlicesProjGPU.cu:211)
//   DD2_gpu_back                        (AAPM_script/MultiSlicesBackGPU.cu:187)
// The multi-GPU split/gather and the mexFunction entries are bypassed: one
// GPU, all slices.  Note the reference calls cudaDeviceReset on every call
// (MultiSlicesProjGPU.cu:217, MultiSlicesBackGPU.cu:196) and exit(1) on CUDA
// errors (utilities.cuh:57-63): run it in a process of its own.
#include <cstdint>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

typedef unsigned char byte;
namespace DD2 {
void DD2_gpu_proj_branchless_sat2d(float x0, float y0, int DNU, float* xds, float* yds,
                                   float imgXCenter, float imgYCenter, float* hangs, int PN,
                                   int XN, int YN, int SLN, float* vol, float* hprj, float dx,
                                   byte* mask, int gpunum);
}
void DD2_gpu_back(float x0, float y0, int DNU, float* xds, float* yds, float detCntIdx,
                  float imgXCenter, float imgYCenter, float* hangs, int PN, int XN, int YN,
                  int SLN, float* hvol, float* hprj, float dx, byte* mask, int gpunum);

extern "C" {
// MATLAB API stand-ins referenced by the (never called) mexFunction entries.
void* mxGetData(const void*) { return nullptr; }
double* mxGetPr(const void*) { return nullptr; }
void* mxCreateNumericArray(size_t, const size_t*, int, int) { return nullptr; }

// Forward projection of vol[YN][XN][SLN] into prj[PN][DNU][SLN] by the reference kernels.
int ddref_proj(float x0, float y0, int DNU, const float* xds, const float* yds,
               float imgXCenter, float imgYCenter, const float* hangs, int PN, int XN, int YN,
               int SLN, const float* vol, float dx, const uint8_t* mask, float* prj) {
  // the reference masks its input in place (MultiSlicesProjGPU.cu:202-209): work on copies
  std::vector<float> v(vol, vol + (size_t)XN * YN * SLN);
  std::vector<float> a(hangs, hangs + (size_t)PN * SLN);
  std::vector<float> xd(xds, xds + DNU), yd(yds, yds + DNU);
  std::vector<byte> m(mask, mask + (size_t)XN * YN);
  DD2::DD2_gpu_proj_branchless_sat2d(x0, y0, DNU, xd.data(), yd.data(), imgXCenter, imgYCenter,
                                     a.data(), PN, XN, YN, SLN, v.data(), prj, dx, m.data(), 0);
  return 0;
}

// Backprojection of prj[PN][DNU][SLN] into vol[YN][XN][SLN] by the reference kernels.
// vol must be zero-filled by the caller: masked voxels are not written by the kernel.
int ddref_back(float x0, float y0, int DNU, const float* xds, const float* yds, float detCntIdx,
               float imgXCenter, float imgYCenter, const float* hangs, int PN, int XN, int YN,
               int SLN, const float* prj, float dx, const uint8_t* mask, float* vol) {
  std::vector<float> p(prj, prj + (size_t)PN * DNU * SLN);
  std::vector<float> a(hangs, hangs + (size_t)PN * SLN);
  std::vector<float> xd(xds, xds + DNU), yd(yds, yds + DNU);
  std::vector<byte> m(mask, mask + (size_t)XN * YN);
  DD2_gpu_back(x0, y0, DNU, xd.data(), yd.data(), detCntIdx, imgXCenter, imgYCenter, a.data(), PN,
               XN, YN, SLN, vol, p.data(), dx, m.data(), 0);
  return 0;
}
}
