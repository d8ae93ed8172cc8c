// Test-infrastructure harness around the reference's byte converters
// (AAPM_script/cov_4uint8_to_float.cpp, cov_8uint8_to_2floats.cpp,
// cov_8uint8_to_double.cpp, cov_uint8_to_double.cpp, cov_uint8_to_PhoStat.cpp),
// compiled unmodified next to this file with their mexFunction renamed (see
// oracle/Makefile).  It supplies the few mx* functions they call and a C entry
// per converter for ctypes.
#include <cstdlib>
#include <cstring>

#include "mex.h"

struct mxArray_tag {
  void* data;
};

extern "C" {
void* mxGetData(const mxArray* a) { return a->data; }
double* mxGetPr(const mxArray* a) { return static_cast<double*>(a->data); }
mxArray* mxCreateNumericArray(mwSize, const mwSize*, mxClassID, mxComplexity) { return nullptr; }
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity) {
  mxArray* a = static_cast<mxArray*>(std::calloc(1, sizeof(mxArray)));
  a->data = std::calloc(m * n ? m * n : 1, sizeof(double));
  return a;
}
}

void ddref_cov_f4(int, mxArray*[], int, const mxArray*[]);
void ddref_cov_2f4(int, mxArray*[], int, const mxArray*[]);
void ddref_cov_d8(int, mxArray*[], int, const mxArray*[]);
void ddref_cov_atof(int, mxArray*[], int, const mxArray*[]);
void ddref_cov_phostat(int, mxArray*[], int, const mxArray*[]);

static void release(mxArray* a) {
  if (!a) return;
  std::free(a->data);
  std::free(a);
}

extern "C" {
double ddref_cov_4uint8_to_float(const unsigned char* b) {
  mxArray in{const_cast<unsigned char*>(b)};
  const mxArray* prhs[1] = {&in};
  mxArray* plhs[1] = {nullptr};
  ddref_cov_f4(1, plhs, 1, prhs);
  const double r = *mxGetPr(plhs[0]);
  release(plhs[0]);
  return r;
}

void ddref_cov_8uint8_to_2floats(const unsigned char* b, double* x, double* y) {
  mxArray in{const_cast<unsigned char*>(b)};
  const mxArray* prhs[1] = {&in};
  mxArray* plhs[2] = {nullptr, nullptr};
  ddref_cov_2f4(2, plhs, 1, prhs);
  *x = *mxGetPr(plhs[0]);
  *y = *mxGetPr(plhs[1]);
  release(plhs[0]);
  release(plhs[1]);
}

double ddref_cov_8uint8_to_double(const unsigned char* b) {
  mxArray in{const_cast<unsigned char*>(b)};
  const mxArray* prhs[1] = {&in};
  mxArray* plhs[1] = {nullptr};
  ddref_cov_d8(1, plhs, 1, prhs);
  const double r = *mxGetPr(plhs[0]);
  release(plhs[0]);
  return r;
}

// b must be NUL-terminated here (MATLAB's uint8 array is not; DICOM pads DS
// strings with a space, where atof stops)
double ddref_cov_uint8_to_double(const char* b) {
  mxArray in{const_cast<char*>(b)};
  const mxArray* prhs[1] = {&in};
  mxArray* plhs[1] = {nullptr};
  ddref_cov_atof(1, plhs, 1, prhs);
  const double r = *mxGetPr(plhs[0]);
  release(plhs[0]);
  return r;
}

void ddref_cov_uint8_to_PhoStat(const unsigned char* b, int n, double* out) {
  mxArray in{const_cast<unsigned char*>(b)};
  mxArray cnt{&n};
  const mxArray* prhs[2] = {&in, &cnt};
  mxArray* plhs[1] = {nullptr};
  ddref_cov_phostat(1, plhs, 2, prhs);
  std::memcpy(out, mxGetPr(plhs[0]), sizeof(double) * (n > 0 ? n : 0));
  release(plhs[0]);
}
}
