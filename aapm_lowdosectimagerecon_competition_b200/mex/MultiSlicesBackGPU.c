/* MultiSlicesBackGPU mex shim over libddfan: the 17 inputs of the reference's
 * mex (AAPM_script/MultiSlicesBackGPU.cu:409-436, called from
 * DD2MutiSlices.m:112-114) in the same order and classes; output
 * single(SLN, XN, YN). */
#include "ddfan_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* fn = "MultiSlicesBackGPU";
  int i;
  (void)nlhs;
  if (nrhs != 17) mexErrMsgTxt("MultiSlicesBackGPU: 17 inputs expected");
  for (i = 0; i < 17; ++i) {
    if (i == 2 || (i >= 9 && i <= 12) || i == 16) DDFAN_MEX_INT32(fn, prhs, i);
    else if (i != 15) DDFAN_MEX_SINGLE(fn, prhs, i);
  }
  {
    const int DNU = ddfan_mex_i(prhs[2]), PN = ddfan_mex_i(prhs[9]);
    const int XN = ddfan_mex_i(prhs[10]), YN = ddfan_mex_i(prhs[11]), SLN = ddfan_mex_i(prhs[12]);
    mwSize dims[3];
    dims[0] = (mwSize)SLN; dims[1] = (mwSize)XN; dims[2] = (mwSize)YN;
    plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
    ddfan_mex_check(ddfan_MultiSlicesBackGPU(
        ddfan_mex_f(prhs[0]), ddfan_mex_f(prhs[1]), DNU, (const float*)mxGetData(prhs[3]),
        (const float*)mxGetData(prhs[4]), ddfan_mex_f(prhs[5]), ddfan_mex_f(prhs[6]), ddfan_mex_f(prhs[7]),
        (const float*)mxGetData(prhs[8]), PN, XN, YN, SLN, (const float*)mxGetData(prhs[13]),
        ddfan_mex_f(prhs[14]), (const uint8_t*)mxGetData(prhs[15]), (const int32_t*)mxGetData(prhs[16]),
        (int)mxGetNumberOfElements(prhs[16]), ddfan_mex_sat_mode(), ddfan_mex_back_mode(),
        (float*)mxGetData(plhs[0])));
  }
}
