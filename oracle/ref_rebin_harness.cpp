// Test-infrastructure harness around the reference's CPU helical-to-fan
// rebinning, HelicalToFan (AAPM_script/HelicalToFanFunc_mex.cpp:142-185),
// compiled unmodified next to this file (see oracle/Makefile).  It only gives
// the function a C entry point for ctypes; mexFunction is compiled but never
// called.  Output layouts are the reference's: Proj [SLN][DefTimes][DetWidth],
// Views [SLN][DefTimes].
#include <cstddef>

void HelicalToFan(float* Proj, float* Views, float* proj, float* zPos, const int SLN, const float SD,
                  const float SO, const float BVAngle, const int DetWidth, const int DetHeight,
                  const float PerDetW, const float PerDetH, const int DefTimes, const float DetCenterW,
                  const float SpiralPitchFactor);

extern "C" {
// MATLAB API stand-ins referenced by the (never called) mexFunction.
void* mxGetData(const void*) { return nullptr; }
double* mxGetPr(const void*) { return nullptr; }
void* mxCreateNumericArray(size_t, const size_t*, int, int) { return nullptr; }

int ddref_helical_to_fan(float* Proj, float* Views, float* proj, float* zPos, int SLN, float SD, float SO,
                         float BVAngle, int DetWidth, int DetHeight, float PerDetW, float PerDetH,
                         int DefTimes, float DetCenterW, float SpiralPitchFactor) {
  HelicalToFan(Proj, Views, proj, zPos, SLN, SD, SO, BVAngle, DetWidth, DetHeight, PerDetW, PerDetH,
               DefTimes, DetCenterW, SpiralPitchFactor);
  return 0;
}
}
