// ddfan_ps.cu -- launchers of the slice-major kernels (per-slice view angles).
#include <algorithm>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_plan.h"
#include "ddfan_ps.h"
#include "ddfan_ps_kernels.cuh"

namespace ddfan {

static int ps_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return DDFAN_OK;
}

int ps_transpose(const float* in, float* out, int B, long long R, int C, cudaStream_t st) {
  if (B < 1 || R < 1 || C < 1) return DDFAN_OK;
  if (B > 65535) return set_err(DDFAN_ERR_UNSUPPORTED, "transpose of %d planes", B);
  const long long nrt = (R + 31) / 32;
  dim3 grid((C + 31) / 32, (unsigned)std::min<long long>(nrt, 65535), B);
  k_ps_transpose<<<grid, 256, 0, st>>>(in, out, R, C);
  return ps_check("k_ps_transpose");
}

template <int M, int C, int KIND>
static void ps_scan_c(const PsScanArgs& a, cudaStream_t st) {
  constexpr int WPC = C > 24 ? 2 : 4;  // warps (lines) per CTA, as k_ps_scan
  k_ps_scan<M, C, KIND><<<(a.nlines + WPC - 1) / WPC, 32 * WPC, 0, st>>>(a);
}

template <int M, int KIND>
static void ps_scan_go(const PsScanArgs& a, cudaStream_t st) {
  const int C = (a.N + 31) / 32;
  if (C <= 8) ps_scan_c<M, 8, KIND>(a, st);
  else if (C <= 16) ps_scan_c<M, 16, KIND>(a, st);
  else if (C <= 24) ps_scan_c<M, 24, KIND>(a, st);
  else ps_scan_c<M, 32, KIND>(a, st);
}

template <int KIND>
static void ps_scan_kind(int mode, const PsScanArgs& a, cudaStream_t st) {
  switch (mode) {
    case SAT_FP32: ps_scan_go<SAT_FP32, KIND>(a, st); break;
    case SAT_HILO: ps_scan_go<SAT_HILO, KIND>(a, st); break;
    default: ps_scan_go<SAT_FP64, KIND>(a, st); break;
  }
}

int ps_scan(int mode, int kind, const PsScanArgs& a, cudaStream_t st) {
  mode = cell_mode(mode);  // these tables keep hi/lo cells in the direct mode
  if (a.N < 1 || a.N > 1024 || a.Nw < a.N + a.pad)
    return set_err(DDFAN_ERR_UNSUPPORTED, "slice-major prefix sums: %d values in %d cells", a.N, a.Nw);
  if (a.nlines < 1) return DDFAN_OK;
  if (kind == 0) ps_scan_kind<0>(mode, a, st);
  else if (kind == 1) ps_scan_kind<1>(mode, a, st);
  else ps_scan_kind<2>(mode, a, st);
  return ps_check("k_ps_scan");
}

int ps_fwd(int mode, const PsFwdArgs& a, int cnt, int Z, cudaStream_t st) {
  mode = cell_mode(mode);  // these tables keep hi/lo cells in the direct mode
  if (cnt < 1 || Z < 1) return DDFAN_OK;
  if (cnt > 65535 || Z > 65535) return set_err(DDFAN_ERR_UNSUPPORTED, "slice-major forward: %d views x %d slices", cnt, Z);
  dim3 grid((a.U + 247) / 248, cnt, Z);
  ProfScope ps(KIND_FWD, st);
  switch (mode) {
    case SAT_FP32: k_ps_fwd<SAT_FP32><<<grid, 256, 0, st>>>(a); break;
    case SAT_HILO: k_ps_fwd<SAT_HILO><<<grid, 256, 0, st>>>(a); break;
    default: k_ps_fwd<SAT_FP64><<<grid, 256, 0, st>>>(a); break;
  }
  return ps_check("k_ps_fwd");
}

int ps_back(int mode, const PsBackArgs& a, int Z, cudaStream_t st) {
  mode = cell_mode(mode);  // these tables keep hi/lo cells in the direct mode
  if (Z < 1) return DDFAN_OK;
  if (Z > 65535) return set_err(DDFAN_ERR_UNSUPPORTED, "slice-major backprojection: %d slices", Z);
  if (a.U + 1 > 1024 || a.M > 4096) return set_err(DDFAN_ERR_UNSUPPORTED, "slice-major backprojection: %d channels", a.U);
  dim3 grid((a.XN + 61) / 62, (a.YN + 4 * kPsBackRows - 1) / (4 * kPsBackRows), Z);
  ProfScope ps(KIND_BACK_A, st);
  switch (mode) {
    case SAT_FP32: k_ps_back_adj<SAT_FP32><<<grid, 256, 0, st>>>(a); break;
    case SAT_HILO: k_ps_back_adj<SAT_HILO><<<grid, 256, 0, st>>>(a); break;
    default: k_ps_back_adj<SAT_FP64><<<grid, 256, 0, st>>>(a); break;
  }
  return ps_check("k_ps_back_adj");
}

int ps_back_ref(int mode, const PsBackArgs& a, int Z, cudaStream_t st) {
  mode = cell_mode(mode);  // these tables keep hi/lo cells in the direct mode
  if (Z < 1) return DDFAN_OK;
  if (Z > 65535) return set_err(DDFAN_ERR_UNSUPPORTED, "slice-major backprojection: %d slices", Z);
  dim3 grid((a.XN + 63) / 64, (a.YN + 4 * kPsRefRows - 1) / (4 * kPsRefRows), Z);
  ProfScope ps(KIND_BACK_A, st);
  switch (mode) {
    case SAT_FP32: k_ps_back_ref<SAT_FP32><<<grid, 256, 0, st>>>(a); break;
    case SAT_HILO: k_ps_back_ref<SAT_HILO><<<grid, 256, 0, st>>>(a); break;
    default: k_ps_back_ref<SAT_FP64><<<grid, 256, 0, st>>>(a); break;
  }
  return ps_check("k_ps_back_ref");
}

}  // namespace ddfan
