/* MultiSlicesProjGPU mex shim over libddfan: the 16 inputs of the reference's
 * mex (AAPM_script/MultiSlicesProjGPU.cu:550-575, called from
 * DD2MutiSlices.m:107-108) in the same order and classes; output
 * single(SLN, DNU, PN). */
#include "ddfan_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* fn = "MultiSlicesProjGPU";
  int i;
  (void)nlhs;
  if (nrhs != 16) mexErrMsgTxt("MultiSlicesProjGPU: 16 inputs expected");
  for (i = 0; i < 16; ++i) {
    if (i == 2 || (i >= 8 && i <= 11) || i == 15) DDFAN_MEX_INT32(fn, prhs, i);
    else if (i != 14) DDFAN_MEX_SINGLE(fn, prhs, i);
  }
  {
    const int DNU = ddfan_mex_i(prhs[2]), PN = ddfan_mex_i(prhs[8]);
    const int XN = ddfan_mex_i(prhs[9]), YN = ddfan_mex_i(prhs[10]), SLN = ddfan_mex_i(prhs[11]);
    mwSize dims[3];
    dims[0] = (mwSize)SLN; dims[1] = (mwSize)DNU; dims[2] = (mwSize)PN;
    plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
    ddfan_mex_check(ddfan_MultiSlicesProjGPU(
        ddfan_mex_f(prhs[0]), ddfan_mex_f(prhs[1]), DNU, (const float*)mxGetData(prhs[3]),
        (const float*)mxGetData(prhs[4]), ddfan_mex_f(prhs[5]), ddfan_mex_f(prhs[6]),
        (const float*)mxGetData(prhs[7]), PN, XN, YN, SLN, (const float*)mxGetData(prhs[12]),
        ddfan_mex_f(prhs[13]), (const uint8_t*)mxGetData(prhs[14]), (const int32_t*)mxGetData(prhs[15]),
        (int)mxGetNumberOfElements(prhs[15]), ddfan_mex_sat_mode(), (float*)mxGetData(plhs[0])));
  }
}
