/* HelicalToFanFunc_mex shim over libddfan: the 13 inputs of the reference's
 * mex (AAPM_script/HelicalToFanFunc_mex.cpp:186-249, called from
 * HelicalToFan_routine.m:39-42) in the same order and classes; outputs
 * single(DetWidth, DefTimes, SLN) and single(DefTimes, SLN).  The raw view
 * count comes from the size of the first input, as in the reference. */
#include "ddfan_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* fn = "HelicalToFanFunc_mex";
  int i;
  (void)nlhs;
  if (nrhs != 13) mexErrMsgTxt("HelicalToFanFunc_mex: 13 inputs expected");
  for (i = 0; i < 13; ++i) {
    if (i == 2 || i == 6 || i == 7 || i == 10) DDFAN_MEX_INT32(fn, prhs, i);
    else DDFAN_MEX_SINGLE(fn, prhs, i);
  }
  {
    const int SLN = ddfan_mex_i(prhs[2]), W = ddfan_mex_i(prhs[6]), H = ddfan_mex_i(prhs[7]);
    const int T = ddfan_mex_i(prhs[10]);
    long long nViews;
    mwSize dp[3], dv[2];
    if (W < 1 || H < 1) mexErrMsgTxt("HelicalToFanFunc_mex: DetWidth and DetHeight must be positive");
    if ((long long)mxGetNumberOfElements(prhs[1]) < SLN) mexErrMsgTxt("HelicalToFanFunc_mex: zPos has fewer than SLN entries");
    nViews = (long long)mxGetNumberOfElements(prhs[0]) / ((long long)W * H);
    dp[0] = (mwSize)W; dp[1] = (mwSize)T; dp[2] = (mwSize)SLN;
    dv[0] = (mwSize)T; dv[1] = (mwSize)SLN;
    plhs[0] = mxCreateNumericArray(3, dp, mxSINGLE_CLASS, mxREAL);
    plhs[1] = mxCreateNumericArray(2, dv, mxSINGLE_CLASS, mxREAL);
    ddfan_mex_check(ddfan_HelicalToFan((float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1]),
                                       (const float*)mxGetData(prhs[0]), nViews, (const float*)mxGetData(prhs[1]),
                                       SLN, ddfan_mex_f(prhs[3]), ddfan_mex_f(prhs[4]), ddfan_mex_f(prhs[5]), W, H,
                                       ddfan_mex_f(prhs[8]), ddfan_mex_f(prhs[9]), T, ddfan_mex_f(prhs[11]),
                                       ddfan_mex_f(prhs[12])));
  }
}
