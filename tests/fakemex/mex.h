/* A stand-in for the part of MATLAB's mex API the shims under
 * aapm_lowdosectimagerecon_competition_b200/mex use, written for the tests:
 * the shims compile against it unchanged and run from Python with arrays
 * that wrap numpy buffers.  Not MATLAB's header.  mexErrMsgTxt unwinds to
 * the caller of fm_call (MATLAB's does not return either). */
#ifndef DDFAN_TEST_FAKEMEX_H
#define DDFAN_TEST_FAKEMEX_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT32_CLASS = 12,
               mxUINT8_CLASS = 9 } mxClassID;
typedef enum { mxREAL = 0 } mxComplexity;
void* mxGetData(const mxArray*);
double* mxGetPr(const mxArray*);
size_t mxGetNumberOfElements(const mxArray*);
int mxIsSingle(const mxArray*);
int mxIsInt32(const mxArray*);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cx);
void mexErrMsgTxt(const char* msg);
#ifdef __cplusplus
}
#endif
#endif
