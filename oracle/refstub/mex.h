/* Minimal stand-in for MATLAB's mex.h, written for this repository.
 * It only lets the reference's MultiSlicesProjGPU.cu / MultiSlicesBackGPU.cu
 * translation units compile as plain CUDA objects; the MATLAB entry points
 * (mexFunction) are compiled but never called.  Test infrastructure only. */
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
#ifdef __cplusplus
}
#endif
#endif
