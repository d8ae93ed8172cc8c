/* Helpers shared by the MATLAB mex shims over libddfan (header-only).
 * Build a shim where MATLAB exists, e.g.
 *   mex -I<repo>/include MultiSlicesProjGPU.c \
 *       -L<repo>/aapm_lowdosectimagerecon_competition_b200 -lddfan
 * The prefix-sum precision and the backprojector follow the environment
 * variables DDFAN_MEX_SAT (fp32 | hilo | fp64, default hilo) and
 * DDFAN_MEX_BACK (ref | adj, default ref: the reference's operator). */
#ifndef DDFAN_MEX_COMMON_H
#define DDFAN_MEX_COMMON_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ddfan.h"
#include "mex.h"

#if defined(__GNUC__)
#define DDFAN_MEX_MAYBE_UNUSED __attribute__((unused))
#else
#define DDFAN_MEX_MAYBE_UNUSED
#endif

DDFAN_MEX_MAYBE_UNUSED static int ddfan_mex_sat_mode(void) {
  const char* v = getenv("DDFAN_MEX_SAT");
  if (v && strcmp(v, "fp32") == 0) return DDFAN_SAT_FP32;
  if (v && strcmp(v, "fp64") == 0) return DDFAN_SAT_FP64;
  return DDFAN_SAT_HILO;
}

DDFAN_MEX_MAYBE_UNUSED static int ddfan_mex_back_mode(void) {
  const char* v = getenv("DDFAN_MEX_BACK");
  return (v && strcmp(v, "adj") == 0) ? DDFAN_BACK_ADJ : DDFAN_BACK_REF;
}

/* Argument checks the reference's mex functions do not make: a wrong class
 * there is read as raw bytes; here it is an error. */
DDFAN_MEX_MAYBE_UNUSED static void ddfan_mex_need(int ok, const char* fn, int idx, const char* what) {
  if (!ok) {
    char msg[160];
    snprintf(msg, sizeof msg, "%s: input %d must be %s", fn, idx + 1, what);
    mexErrMsgTxt(msg);
  }
}

#define DDFAN_MEX_SINGLE(fn, prhs, i) ddfan_mex_need(mxIsSingle(prhs[i]), fn, i, "single")
#define DDFAN_MEX_INT32(fn, prhs, i) ddfan_mex_need(mxIsInt32(prhs[i]), fn, i, "int32")

DDFAN_MEX_MAYBE_UNUSED static float ddfan_mex_f(const mxArray* a) { return *(const float*)mxGetData(a); }
DDFAN_MEX_MAYBE_UNUSED static int ddfan_mex_i(const mxArray* a) { return *(const int*)mxGetData(a); }

DDFAN_MEX_MAYBE_UNUSED static void ddfan_mex_check(int rc) {
  if (rc != DDFAN_OK) mexErrMsgTxt(ddfan_last_error());
}

#endif
