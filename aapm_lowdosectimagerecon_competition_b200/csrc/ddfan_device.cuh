// ddfan_device.cuh -- device-side building blocks shared by the ddfan kernels.
//
// Prefix-sum ("SAT") cells.  A table is a 3-D array of cells [line][k][zb]:
// `line` is the image row/column (or the view, for sinogram tables), k the
// position along the line, zb a block of 4 consecutive slices.  Within a row
// (line, k) the z-blocks are grouped in z-tiles of ZL blocks and each tile
// stores its cells plane by plane (all S_hi of the tile, then all S_lo, then
// all v), so the ZL lanes that own a tile read each plane as one contiguous
// ZL*16-byte run: float4 index of plane j of block zb in row r is
//   (r * ZBp + (zb / ZL) * ZL) * F4 + j * ZL + zb % ZL,  ZBp = ZB rounded up to ZL.  A cell holds,
// for its 4 slices, the exclusive prefix sum S[k] = sum_{j<k} v[j] and the
// value v[k] itself, so a linearly interpolated prefix sum at position
// c in [k, k+1] is S[k] + (c - k) v[k]: one cell per sample.  This is the
// zero-padded summed-area table of the reference (AAPM_script/
// MultiSlicesProjGPU.cu:25-51, MultiSlicesBackGPU.cu:12-32) sampled the way
// its linear-filtered, clamped textures sample it, with exact weights.
//
//   DDFAN_SAT_FP32  cell = {float4 S, float4 v}                 32 B
//   DDFAN_SAT_HILO  cell = {float4 S_hi, float4 S_lo, float4 v} 48 B
//   DDFAN_SAT_FP64  cell = {double4 S, float4 v}                48 B
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ddfan {

constexpr int SAT_FP32 = 0, SAT_HILO = 1, SAT_FP64 = 2;
// no prefix-sum tables: footprint differences read the values directly (ddfan_dd_kernels.cuh)
constexpr int SAT_DIRECT = 3;

// the cell format that stands in for SAT_DIRECT where a path keeps tables
__host__ __device__ inline int cell_mode(int mode) { return mode == SAT_DIRECT ? SAT_HILO : mode; }

template <int M> struct CellInfo;
template <> struct CellInfo<SAT_FP32> { static constexpr int F4 = 2; };
template <> struct CellInfo<SAT_HILO> { static constexpr int F4 = 3; };
template <> struct CellInfo<SAT_FP64> { static constexpr int F4 = 3; };

__host__ __device__ inline int cell_f4(int mode) { return mode == SAT_FP32 ? 2 : 3; }

// ---------------------------------------------------------------- error-free sums

// Knuth's TwoSum: s + e == a + b exactly (round-to-nearest, no reassociation).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  float bp = __fsub_rn(s, a);
  float ap = __fsub_rn(s, bp);
  e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}

// Running compensated sum of 4 slices.
template <int M> struct Acc4;

template <> struct Acc4<SAT_FP32> {
  float s[4];
  __device__ void zero() { s[0] = s[1] = s[2] = s[3] = 0.f; }
  __device__ void add(const float (&v)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = __fadd_rn(s[i], v[i]);
  }
  __device__ void add(const Acc4& o) {
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = __fadd_rn(s[i], o.s[i]);
  }
  __device__ Acc4 shfl_up(int off) const {
    Acc4 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) r.s[i] = __shfl_up_sync(0xffffffffu, s[i], off);
    return r;
  }
  __device__ void store(float4* cell, int ps, const float (&v)[4]) const {
    cell[0] = make_float4(s[0], s[1], s[2], s[3]);
    cell[ps] = make_float4(v[0], v[1], v[2], v[3]);
  }
};

template <> struct Acc4<SAT_HILO> {
  float hi[4], lo[4];
  __device__ void zero() {
#pragma unroll
    for (int i = 0; i < 4; ++i) hi[i] = lo[i] = 0.f;
  }
  __device__ void add(const float (&v)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float s, e;
      two_sum(hi[i], v[i], s, e);
      hi[i] = s;
      lo[i] = __fadd_rn(lo[i], e);
    }
  }
  __device__ void add(const Acc4& o) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float s, e;
      two_sum(hi[i], o.hi[i], s, e);
      hi[i] = s;
      lo[i] = __fadd_rn(__fadd_rn(lo[i], o.lo[i]), e);
    }
  }
  __device__ Acc4 shfl_up(int off) const {
    Acc4 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      r.hi[i] = __shfl_up_sync(0xffffffffu, hi[i], off);
      r.lo[i] = __shfl_up_sync(0xffffffffu, lo[i], off);
    }
    return r;
  }
  // stores the renormalised pair (hi = fl(hi + lo)) so hi differences are clean
  __device__ void store(float4* cell, int ps, const float (&v)[4]) const {
    float h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float s = __fadd_rn(hi[i], lo[i]);
      l[i] = __fsub_rn(lo[i], __fsub_rn(s, hi[i]));
      h[i] = s;
    }
    cell[0] = make_float4(h[0], h[1], h[2], h[3]);
    cell[ps] = make_float4(l[0], l[1], l[2], l[3]);
    cell[2 * ps] = make_float4(v[0], v[1], v[2], v[3]);
  }
};

template <> struct Acc4<SAT_FP64> {
  double s[4];
  __device__ void zero() { s[0] = s[1] = s[2] = s[3] = 0.0; }
  __device__ void add(const float (&v)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = __dadd_rn(s[i], (double)v[i]);
  }
  __device__ void add(const Acc4& o) {
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = __dadd_rn(s[i], o.s[i]);
  }
  __device__ Acc4 shfl_up(int off) const {
    Acc4 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) r.s[i] = __shfl_up_sync(0xffffffffu, s[i], off);
    return r;
  }
  __device__ void store(float4* cell, int ps, const float (&v)[4]) const {
    *reinterpret_cast<double2*>(cell) = make_double2(s[0], s[1]);
    *reinterpret_cast<double2*>(cell + ps) = make_double2(s[2], s[3]);
    cell[2 * ps] = make_float4(v[0], v[1], v[2], v[3]);
  }
};

// ---------------------------------------------------------------- interpolation

// Interpolated prefix sum Phi = S[k] + f v[k] for 4 slices, kept in the
// table's precision so that differences of two samples do not cancel.
template <int M> struct Phi4;

template <> struct Phi4<SAT_FP32> {
  float v[4];
  __device__ __forceinline__ void load(const float4* cell, int ps, float f) {
    float4 s = __ldg(cell), p = __ldg(cell + ps);
    v[0] = fmaf(f, p.x, s.x); v[1] = fmaf(f, p.y, s.y);
    v[2] = fmaf(f, p.z, s.z); v[3] = fmaf(f, p.w, s.w);
  }
  __device__ __forceinline__ void zero() { v[0] = v[1] = v[2] = v[3] = 0.f; }
  // this - o
  __device__ __forceinline__ void diff(const Phi4& o, float (&d)[4]) const {
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = v[i] - o.v[i];
  }
};

template <> struct Phi4<SAT_HILO> {
  float hi[4], lo[4];
  __device__ __forceinline__ void load(const float4* cell, int ps, float f) {
    float4 h = __ldg(cell), l = __ldg(cell + ps), p = __ldg(cell + 2 * ps);
    hi[0] = h.x; hi[1] = h.y; hi[2] = h.z; hi[3] = h.w;
    lo[0] = fmaf(f, p.x, l.x); lo[1] = fmaf(f, p.y, l.y);
    lo[2] = fmaf(f, p.z, l.z); lo[3] = fmaf(f, p.w, l.w);
  }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < 4; ++i) hi[i] = lo[i] = 0.f;
  }
  __device__ __forceinline__ void diff(const Phi4& o, float (&d)[4]) const {
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = __fadd_rn(__fsub_rn(hi[i], o.hi[i]), __fsub_rn(lo[i], o.lo[i]));
  }
};

template <> struct Phi4<SAT_FP64> {
  double v[4];
  __device__ __forceinline__ void load(const float4* cell, int ps, float f) {
    double2 a = __ldg(reinterpret_cast<const double2*>(cell));
    double2 b = __ldg(reinterpret_cast<const double2*>(cell + ps));
    float4 p = __ldg(cell + 2 * ps);
    const double fd = (double)f;
    v[0] = fma(fd, (double)p.x, a.x); v[1] = fma(fd, (double)p.y, a.y);
    v[2] = fma(fd, (double)p.z, b.x); v[3] = fma(fd, (double)p.w, b.y);
  }
  __device__ __forceinline__ void zero() { v[0] = v[1] = v[2] = v[3] = 0.0; }
  __device__ __forceinline__ void diff(const Phi4& o, float (&d)[4]) const {
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = (float)(v[i] - o.v[i]);
  }
};

// ---------------------------------------------------------------- per-view geometry

// Per-view constants written by k_view_geom (one entry per view of a call).
struct ViewGeom {
  double cs, sn;    // cos / sin of the wrapped view angle
  double sx, sy;    // source position
  float shx, shy;   // unit vector source -> rotation centre
  float sgn;        // sign of d(line coordinate)/d(boundary index) (exact adjoint)
  int xmajor;       // |cos| <= |sin|: rays are integrated column by column (x lines)
};

}  // namespace ddfan
