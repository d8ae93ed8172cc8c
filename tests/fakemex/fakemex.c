/* Implementation of tests/fakemex/mex.h plus the entry points the tests call
 * through ctypes (fm_wrap, fm_call, fm_data, fm_dims, fm_free). */
#include <setjmp.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  size_t n, ndim, dims[8];
  void* data;
  int owned;
};

static jmp_buf g_jmp;
static char g_err[512];

static size_t class_bytes(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: return 4;
    case mxUINT8_CLASS: return 1;
    default: return 1;
  }
}

void* mxGetData(const mxArray* a) { return a->data; }
double* mxGetPr(const mxArray* a) { return (double*)a->data; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->n; }
int mxIsSingle(const mxArray* a) { return a->cls == mxSINGLE_CLASS; }
int mxIsInt32(const mxArray* a) { return a->cls == mxINT32_CLASS; }

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cx) {
  (void)cx;
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = cls;
  a->ndim = ndim;
  a->n = 1;
  for (size_t i = 0; i < ndim && i < 8; ++i) {
    a->dims[i] = dims[i];
    a->n *= dims[i];
  }
  a->data = calloc(a->n ? a->n : 1, class_bytes(cls));
  a->owned = 1;
  return a;
}

void mexErrMsgTxt(const char* msg) {
  strncpy(g_err, msg ? msg : "", sizeof g_err - 1);
  g_err[sizeof g_err - 1] = 0;
  longjmp(g_jmp, 1);
}

/* an array over a caller-owned buffer (numpy), MATLAB dims */
mxArray* fm_wrap(int cls, size_t ndim, const size_t* dims, void* data) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = (mxClassID)cls;
  a->ndim = ndim;
  a->n = 1;
  for (size_t i = 0; i < ndim && i < 8; ++i) {
    a->dims[i] = dims[i];
    a->n *= dims[i];
  }
  a->data = data;
  return a;
}

void* fm_data(mxArray* a) { return a->data; }
size_t fm_numel(mxArray* a) { return a->n; }
void fm_free(mxArray* a) {
  if (!a) return;
  if (a->owned) free(a->data);
  free(a);
}

typedef void (*mexfn)(int, mxArray**, int, const mxArray**);

/* runs mexFunction; returns 0, or 1 with the error text in msg */
int fm_call(mexfn f, int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs, char* msg, size_t cap) {
  if (setjmp(g_jmp)) {
    if (msg && cap) {
      strncpy(msg, g_err, cap - 1);
      msg[cap - 1] = 0;
    }
    return 1;
  }
  f(nlhs, plhs, nrhs, prhs);
  return 0;
}
