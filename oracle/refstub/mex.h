/* Minimal stand-in for MATLAB's mex.h, written for this repository.
 * It only lets the reference's MultiSlicesProjGPU.cu / MultiSlicesBackGPU.cu /
 * HelicalToFanFunc_mex.cpp translation units compile as plain objects (their
 * mexFunction is compiled but never called) and the reference's cov_*.cpp
 * byte converters run through oracle/ref_cov_harness.cpp.  Test
 * infrastructure only. */
#ifndef DDFAN_REFSTUB_MEX_H
#define DDFAN_REFSTUB_MEX_H
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0 } mxComplexity;
#ifdef __cplusplus
extern "C" {
#endif
void* mxGetData(const mxArray*);
double* mxGetPr(const mxArray*);
mxArray* mxCreateNumericArray(mwSize, const mwSize*, mxClassID, mxComplexity);
mxArray* mxCreateDoubleMatrix(mwSize, mwSize, mxComplexity);
#ifdef __cplusplus
}
#endif
#endif
