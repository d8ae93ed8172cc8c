// ddfan_ps.h -- the slice-major path's launch arguments and launchers
// (kernels in ddfan_ps_kernels.cuh, launchers in ddfan_ps.cu), shared by the
// OS-SART solver and the plans' per-slice-angle entry points.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "ddfan_device.cuh"

namespace ddfan {

// What a slice-major table is built from: lines of an image (one slice's rows
// or columns) or the OS-SART residual of one (slice, view) of a subset.
struct PsScanArgs {
  void* tab;            // cells (PsCell<M>::T), line t at [t * Nw, t * Nw + Nw)
  int nlines, N, Nw;    // lines, values per line, cells per line (Nw >= N + pad; cells past the values hold the total)
  int pad;              // zero cells before the values (image tables: 1, the guard cell of clamped samples)
  // kind 0: src [nlines][N] (slice-major, lines of a slice contiguous), times the
  // image mask [YN][XN] if given; kind 2: src times the weight wgt [nlines][N] * wscale
  const float* src;
  const uint8_t* mask;
  int XN, lines_per_slice, cols;  // cols: line = x column, k = y (mask index k * XN + line)
  // residual: line = z * cnt + m, table line z * cstride + m; y [Z][P][U]
  // (views in the caller's order), ax [Z][cstride][U], rows [(roff + m)][U]
  // (subset order), wgt [Z][cstride][U] or null
  const float* y;
  const float* ax;
  const float* rows;
  const float* wgt;
  float wscale;
  int cnt, cstride, P, roff, ksub, nOS;
};

struct PsFwdArgs {
  const void* tabx;   // image rows [Z][YN][XN + 2] cells (y-major views), guard cell first and last
  const void* taby;   // image columns [Z][XN][YN + 2] cells (x-major views)
  const ViewGeom* vg;   // rows z * cstride + m
  const double2* fc;    // [rows][U+1] boundary lines
  const float* cvd;     // [rows][U]
  float* out;           // [Z][cstride][U]
  int cstride, U, XN, YN;
  float dx;
};

struct PsBackArgs {
  const void* sq;       // weighted residual table [Z][cstride][U+1] cells
  const ViewGeom* vg;
  const double2* fc;
  const float* tb;      // plan's boundary fan tangents (U+1) and bracket lookup (M)
  const uint16_t* lut;
  float t0, invdt, dirt;
  int M;
  int cnt, cstride, U, XN, YN;
  double ocx, ocy, dx;
  double inv_sid, inv_dbeta, cnt_ref;  // REF formula: 1/|source|, 1/(channel angle), detCntIdx + 0.5
  // OS-SART update of x [Z][YN][XN] in place: x += t / colSum where colSum != 0,
  // else x += t, t the masked backprojection; or, with x null, out = t
  float* x;
  const float* colsum;
  int nonneg;
  float* out;
  const uint8_t* mask;
};

// rows of pixels per warp in k_ps_back_adj (8 warps: 2 across x, 4 down y)
constexpr int kPsBackRows = 8;
// and in k_ps_back_ref, whose full FP64 angle is taken on a warp's first row
#ifndef DDFAN_PS_REF_ROWS
#define DDFAN_PS_REF_ROWS 8
#endif
constexpr int kPsRefRows = DDFAN_PS_REF_ROWS;

// out[b][c][r] = in[b][r][c] for b < B, r < R, c < C
int ps_transpose(const float* in, float* out, int B, long long R, int C, cudaStream_t st);
// kind 0: image lines (masked); kind 1: OS-SART residual lines; kind 2: weighted lines
int ps_scan(int mode, int kind, const PsScanArgs& a, cudaStream_t st);
// grid: 31-channel groups x cnt views x Z slices
int ps_fwd(int mode, const PsFwdArgs& a, int cnt, int Z, cudaStream_t st);
int ps_back(int mode, const PsBackArgs& a, int Z, cudaStream_t st);
// the reference backprojector's formula (k_back_ref) in slice-major layout
int ps_back_ref(int mode, const PsBackArgs& a, int Z, cudaStream_t st);

}  // namespace ddfan
