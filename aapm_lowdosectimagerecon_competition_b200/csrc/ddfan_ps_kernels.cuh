// ddfan_ps_kernels.cuh -- kernels for per-slice view angles in slice-major
// layout (the OS-SART solver's "slice-major" path).
//
// The 4-slice cells of ddfan_device.cuh share one gather index, so the four
// slices of a cell must share view geometry.  When every slice has its own
// angle list (helical rebinning, AAPM_script/HelicalToFanFunc_mex.cpp:77-81)
// that sharing is lost; these kernels give each slice its own geometry and
// put the parallelism along the line instead: lanes of a warp own consecutive
// detector boundaries (forward) or consecutive pixels (backprojection), so a
// warp's gathers hit consecutive cells of one slice's line.
//
// Slice-major prefix-sum table: cells [line][k] of every slice, lines of a
// slice contiguous ([z][line][k]), one interleaved cell per (line, k):
//   DDFAN_SAT_FP32  float2 {S, v}
//   DDFAN_SAT_HILO  float4 {S_hi, S_lo, v, 0}
//   DDFAN_SAT_FP64  16 bytes {double S, float v, 0}
// with S[k] the exclusive prefix sum and v[k] the value, as in the 4-slice
// cells: the interpolated prefix sum at c in [k, k+1] is S[k] + (c - k) v[k],
// one 8- or 16-byte load per sample.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ddfan_device.cuh"
#include "ddfan_ps.h"

namespace ddfan {

// ---------------------------------------------------------------- one-slice cells

template <int M> struct PsCell { using T = float4; };
template <> struct PsCell<SAT_FP32> { using T = float2; };

template <int M> struct PhiS;

template <> struct PhiS<SAT_FP32> {
  float v;
  __device__ __forceinline__ void load(const float2* c, float f) {
    const float2 q = __ldg(c);
    v = fmaf(f, q.y, q.x);
  }
  __device__ __forceinline__ PhiS down() const {
    PhiS r;
    r.v = __shfl_down_sync(0xffffffffu, v, 1);
    return r;
  }
  // this - o
  __device__ __forceinline__ float diff(const PhiS& o) const { return v - o.v; }
};

template <> struct PhiS<SAT_HILO> {
  float hi, lo;
  __device__ __forceinline__ void load(const float4* c, float f) {
    const float4 q = __ldg(c);
    hi = q.x;
    lo = fmaf(f, q.z, q.y);
  }
  __device__ __forceinline__ PhiS down() const {
    PhiS r;
    r.hi = __shfl_down_sync(0xffffffffu, hi, 1);
    r.lo = __shfl_down_sync(0xffffffffu, lo, 1);
    return r;
  }
  __device__ __forceinline__ float diff(const PhiS& o) const {
    return __fadd_rn(__fsub_rn(hi, o.hi), __fsub_rn(lo, o.lo));
  }
};

template <> struct PhiS<SAT_FP64> {
  double v;
  __device__ __forceinline__ void load(const float4* c, float f) {
    const float4 q = __ldg(c);
    const double S = __hiloint2double(__float_as_int(q.y), __float_as_int(q.x));
    v = fma((double)f, (double)q.z, S);
  }
  __device__ __forceinline__ PhiS down() const {
    PhiS r;
    r.v = __shfl_down_sync(0xffffffffu, v, 1);
    return r;
  }
  __device__ __forceinline__ float diff(const PhiS& o) const { return (float)(v - o.v); }
};

// Running sum of one slice, with the arithmetic of Acc4.
template <int M> struct AccS;

template <> struct AccS<SAT_FP32> {
  float s;
  __device__ __forceinline__ void zero() { s = 0.f; }
  __device__ __forceinline__ void add(float v) { s = __fadd_rn(s, v); }
  __device__ __forceinline__ void add(const AccS& o) { s = __fadd_rn(s, o.s); }
  __device__ __forceinline__ AccS up(int off) const {
    AccS r;
    r.s = __shfl_up_sync(0xffffffffu, s, off);
    return r;
  }
  // the prefix-sum words of a cell: word j at buf[j * NB + i]
  __device__ __forceinline__ void put(float* buf, int NB, int i) const { buf[i] = s; }
  __device__ __forceinline__ static float2 cell(const float* buf, int NB, int i, float v) {
    return make_float2(buf[i], v);
  }
  __device__ __forceinline__ AccS bcast(int src) const {
    AccS r;
    r.s = __shfl_sync(0xffffffffu, s, src);
    return r;
  }
  __device__ __forceinline__ float2 cell(float v) const { return make_float2(s, v); }
};

template <> struct AccS<SAT_HILO> {
  float hi, lo;
  __device__ __forceinline__ void zero() { hi = lo = 0.f; }
  __device__ __forceinline__ void add(float v) {
    float s, e;
    two_sum(hi, v, s, e);
    hi = s;
    lo = __fadd_rn(lo, e);
  }
  __device__ __forceinline__ void add(const AccS& o) {
    float s, e;
    two_sum(hi, o.hi, s, e);
    hi = s;
    lo = __fadd_rn(__fadd_rn(lo, o.lo), e);
  }
  __device__ __forceinline__ AccS up(int off) const {
    AccS r;
    r.hi = __shfl_up_sync(0xffffffffu, hi, off);
    r.lo = __shfl_up_sync(0xffffffffu, lo, off);
    return r;
  }
  // the renormalised pair (hi = fl(hi + lo)), as Acc4 stores it
  __device__ __forceinline__ void put(float* buf, int NB, int i) const {
    const float s = __fadd_rn(hi, lo);
    buf[i] = s;
    buf[NB + i] = __fsub_rn(lo, __fsub_rn(s, hi));
  }
  __device__ __forceinline__ static float4 cell(const float* buf, int NB, int i, float v) {
    return make_float4(buf[i], buf[NB + i], v, 0.f);
  }
  __device__ __forceinline__ AccS bcast(int src) const {
    AccS r;
    r.hi = __shfl_sync(0xffffffffu, hi, src);
    r.lo = __shfl_sync(0xffffffffu, lo, src);
    return r;
  }
  __device__ __forceinline__ float4 cell(float v) const {
    const float s = __fadd_rn(hi, lo);
    return make_float4(s, __fsub_rn(lo, __fsub_rn(s, hi)), v, 0.f);
  }
};

template <> struct AccS<SAT_FP64> {
  double s;
  __device__ __forceinline__ void zero() { s = 0.0; }
  __device__ __forceinline__ void add(float v) { s = __dadd_rn(s, (double)v); }
  __device__ __forceinline__ void add(const AccS& o) { s = __dadd_rn(s, o.s); }
  __device__ __forceinline__ AccS up(int off) const {
    AccS r;
    r.s = __shfl_up_sync(0xffffffffu, s, off);
    return r;
  }
  __device__ __forceinline__ void put(float* buf, int NB, int i) const {
    buf[i] = __int_as_float(__double2loint(s));
    buf[NB + i] = __int_as_float(__double2hiint(s));
  }
  __device__ __forceinline__ static float4 cell(const float* buf, int NB, int i, float v) {
    return make_float4(buf[i], buf[NB + i], v, 0.f);
  }
  __device__ __forceinline__ AccS bcast(int src) const {
    AccS r;
    r.s = __shfl_sync(0xffffffffu, s, src);
    return r;
  }
  __device__ __forceinline__ float4 cell(float v) const {
    return make_float4(__int_as_float(__double2loint(s)), __int_as_float(__double2hiint(s)), v, 0.f);
  }
};

// 32-bit words of a cell's prefix sum
template <int M> struct PsInfo { static constexpr int SW = M == SAT_FP32 ? 1 : 2; };

// Reciprocal of the footprint length and of the bracket width: the PTX
// approximate reciprocal (at most 1 ulp from the correctly rounded one, per
// the PTX ISA).  __frcp_rn in its place measured 30 % slower on the per-slice
// c3 solve (3.09 -> 2.36 iterations/s); a 768-pixel-line test against the
// FP64 oracle holds the 2e-6 bound with this one.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The REF backprojector's angle step with a Newton reciprocal in place of
// the FP64 division (1: per-slice c3 iteration 365 -> 355 ms of REF
// backprojection) or the division (0)
#ifndef DDFAN_PS_REF_NEWTON
#define DDFAN_PS_REF_NEWTON 1
#endif

// The REF backprojector's channel coordinates in 32.32 fixed point (1: two
// conversions per pixel and view instead of six, which took the per-slice c3
// iteration's REF backprojection from 355 to 314 ms) or FP64 with float
// conversions (0)
#ifndef DDFAN_PS_REF_FIXED
#define DDFAN_PS_REF_FIXED 1
#endif

// ---------------------------------------------------------------- transposes

// out[b][c][r] = in[b][r][c] for b < B, r < R, c < C: 32 x 32 tiles through
// shared memory, both sides coalesced.
static __global__ void __launch_bounds__(256) k_ps_transpose(const float* __restrict__ in, float* __restrict__ out,
                                                             long long R, int C) {
  __shared__ float tile[32][33];
  const size_t plane = (size_t)R * C;
  const float* src = in + blockIdx.z * plane;
  float* dst = out + blockIdx.z * plane;
  const int c0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const long long nrt = (R + 31) / 32;
  for (long long rt = blockIdx.y; rt < nrt; rt += gridDim.y) {  // uniform per CTA
    const long long r0 = rt * 32;
    for (int j = ty; j < 32; j += 8) {
      const long long r = r0 + j;
      const int c = c0 + tx;
      if (r < R && c < C) tile[j][tx] = __ldg(src + (size_t)r * C + c);
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
      const int c = c0 + j;
      const long long r = r0 + tx;
      if (r < R && c < C) dst[(size_t)c * R + r] = tile[tx][j];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- prefix sums

template <int KIND>
__device__ __forceinline__ float ps_value(const PsScanArgs& a, int line, int k) {
  if (k >= a.N) return 0.f;
  if (KIND == 0) {
    const size_t e = (size_t)line * a.N + k;
    float v = __ldg(a.src + e);
    if (a.mask) {
      const int l = line % a.lines_per_slice;
      v *= (float)a.mask[a.cols ? (size_t)k * a.XN + l : (size_t)l * a.XN + k];
    }
    return v;
  } else if (KIND == 2) {
    const size_t e = (size_t)line * a.N + k;
    return __ldg(a.src + e) * (__ldg(a.wgt + e) * a.wscale);
  } else {
    // r = (y - A x) / rowSum where rowSum != 0, else A x (AAPM_script/OSSART_AAPM.m:86-88),
    // times the channel weight
    const int z = line / a.cnt, m = line - z * a.cnt;
    const int ib = a.ksub + m * a.nOS;
    const size_t row = (size_t)z * a.cstride + m;
    const float rs = __ldg(a.rows + (size_t)(a.roff + m) * a.N + k);
    float v = __ldg(a.ax + row * a.N + k);
    if (rs != 0.f) v = __fdiv_rn(__fsub_rn(__ldg(a.y + ((size_t)z * a.P + ib) * a.N + k), v), rs);
    const float w = a.wgt ? __ldg(a.wgt + row * a.N + k) * a.wscale : a.wscale;
    return v * w;
  }
}

// One warp per line, WPC warps per CTA.  Lane L owns the chunk
// [L*C, L*C + C) of the line's N values (32 C >= N); values go through shared
// memory both ways so that global reads and cell writes are coalesced.  Chunk
// sums are combined by a warp-shuffle exclusive scan.  Cells: pad zero cells,
// the N value cells, then cells holding the total up to Nw.
template <int M, int C, int KIND>
__global__ void __launch_bounds__(128) k_ps_scan(PsScanArgs a) {
  constexpr int WPC = C > 24 ? 2 : 4;
  constexpr int NB = 32 * (C + 1);  // slots per word (chunk j of lane L at L * (C + 1) + j)
  constexpr int SW = PsInfo<M>::SW;
  using Cell = typename PsCell<M>::T;
  __shared__ float sbuf[WPC][(SW + 1) * NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int line = blockIdx.x * WPC + w;
  if (w >= WPC || line >= a.nlines) return;  // uniform per warp; no block-wide barrier below
  float* buf = sbuf[w];
  float* vbuf = buf + SW * NB;
  int tline = line;
  if (KIND == 1) {
    const int z = line / a.cnt;
    tline = z * a.cstride + (line - z * a.cnt);
  }
  Cell* out = reinterpret_cast<Cell*>(a.tab) + (size_t)tline * a.Nw;
  Cell* vout = out + a.pad;
  auto slot = [](int e) { return (e / C) * (C + 1) + e % C; };
  for (int e = lane; e < 32 * C; e += 32) vbuf[slot(e)] = ps_value<KIND>(a, line, e);
  __syncwarp();
  float v[C];
  AccS<M> acc;
  acc.zero();
#pragma unroll
  for (int j = 0; j < C; ++j) {
    v[j] = vbuf[lane * (C + 1) + j];
    acc.add(v[j]);
  }
  AccS<M> inc = acc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const AccS<M> o = inc.up(off);
    if (lane >= off) inc.add(o);
  }
  AccS<M> run = inc.up(1);
  if (lane == 0) run.zero();
#pragma unroll
  for (int j = 0; j < C; ++j) {
    run.put(buf, NB, lane * (C + 1) + j);
    run.add(v[j]);
  }
  const AccS<M> total = run.bcast(31);
  __syncwarp();
  for (int e = lane; e < a.N; e += 32) vout[e] = AccS<M>::cell(buf, NB, slot(e), vbuf[slot(e)]);
  if (lane < a.pad) {
    AccS<M> zero;
    zero.zero();
    out[lane] = zero.cell(0.f);
  }
  for (int e = a.N + a.pad + lane; e < a.Nw; e += 32) out[e] = total.cell(0.f);
}

// ---------------------------------------------------------------- forward

// Branchless DD forward projection (AAPM_script/MultiSlicesProjGPU.cu:100-200)
// of one slice and one of its views per (blockIdx.z, blockIdx.y).  Lane L of
// warp w owns boundary b = (tile * 8 + w) * 31 + L; channel b (lanes 0..30)
// takes (Phi(c_{b+1}) - Phi(c_b)) / length from its neighbour lane, on every
// line, summing chunks of 16 lines into a fresh partial as k_fwd does.  The
// boundary position c_b(ii) = ii F + C runs in 32.32 fixed point from the FP64
// line (error below 1e-7 cells over 1024 lines); the footprint length
// (c_{b+1} - c_b) dx is linear in ii and runs in FP32.  Positions outside the
// line clamp to its guard cells (prefix sum 0 before, the total after, value
// 0), which reproduces k_fwd's clamp of c to [0, N].
template <int M>
__global__ void __launch_bounds__(256) k_ps_fwd(PsFwdArgs a) {
  constexpr int CC = 16, CPW = 31;
  using Cell = typename PsCell<M>::T;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int bw = (blockIdx.x * 8 + w) * CPW;
  if (bw >= a.U) return;  // uniform per warp
  const int m = blockIdx.y, z = blockIdx.z;
  const size_t r = (size_t)z * a.cstride + m;
  const int b = bw + lane;
  const bool xm = a.vg[r].xmajor != 0;
  const int nl = xm ? a.XN : a.YN, N = xm ? a.YN : a.XN;
  const int Nw = N + 2;
  const Cell* line = reinterpret_cast<const Cell*>(xm ? a.taby : a.tabx) + (size_t)z * nl * Nw;
  const double2 f0 = __ldg(a.fc + r * (a.U + 1) + min(b, a.U));
  const double2 f1 = __ldg(a.fc + r * (a.U + 1) + min(b + 1, a.U));
  const double two32 = 4294967296.0;
  const long long dcf = __double2ll_rn(f0.x * two32);
  long long cf = __double2ll_rn(f0.y * two32);
  const float dx = a.dx;
  const float lF = (float)((f1.x - f0.x) * (double)dx), lC = (float)((f1.y - f0.y) * (double)dx);
  float fi = 0.f;
  float acc = 0.f;
  for (int ii0 = 0; ii0 < nl; ii0 += CC) {
    const int ncol = min(CC, nl - ii0);
    float part = 0.f;
#pragma unroll 4
    for (int col = 0; col < ncol; ++col) {
      const int i0 = min(max((int)(cf >> 32), -1), N) + 1;
      const float f = __int_as_float(0x3f800000 | ((unsigned)cf >> 9)) - 1.f;
      PhiS<M> cur;
      cur.load(line + i0, f);
      const PhiS<M> nxt = cur.down();
      part = fmaf(nxt.diff(cur), rcp_approx(fmaf(fi, lF, lC)), part);
      cf += dcf;
      fi += 1.f;
      line += Nw;
    }
    acc += part;
  }
  if (lane < CPW && b < a.U) a.out[r * a.U + b] = acc * (__ldg(a.cvd + r * a.U + b) * dx);
}

// ---------------------------------------------------------------- exact adjoint

// Exact transpose of k_ps_fwd, both view orientations in one pass.  Warp =
// 31 consecutive pixels of a row (lanes 0..30) x R rows of one slice; it
// loops over the slice's views of the subset.  A view integrated along x
// columns (x-major) samples each lane's column at the R + 1 row edges; a view
// integrated along y rows samples each row at the 32 column edges of the warp
// and differences neighbouring lanes.  The sample at a pixel edge (line li,
// edge ck) is the weighted channel prefix sum Q at the edge's fractional
// boundary index b + (ck - c_b(li)) / (c_{b+1}(li) - c_b(li)), c_b the FP64
// boundary lines of the forward.  Each lane guesses the bracket of its first
// edge of a view from the edge's fan tangent (the lookup table of k_back_adj)
// and then walks: it keeps c_b and c_{b+1} at its current line and steps b
// until the edge lies between them -- boundary rays do not cross inside
// the image, so s c_b(li) increases with b on every line (s = the view's sgn);
// the walk runs on s-scaled positions.
template <int M>
__global__ void __launch_bounds__(256) k_ps_back_adj(PsBackArgs a) {
  constexpr int R = kPsBackRows, PX = 31;
  constexpr int LUTMAX = 4096;
  using Cell = typename PsCell<M>::T;
  __shared__ uint16_t s_lut[LUTMAX];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < a.M; i += 256) s_lut[i] = a.lut[i];
  __syncthreads();
  const int z = blockIdx.z;
  const int x0 = (blockIdx.x * 2 + (w & 1)) * PX, y0 = (blockIdx.y * 4 + (w >> 1)) * R;
  if (x0 >= a.XN || y0 >= a.YN) return;  // uniform per warp; no barrier below
  const float tfirst = __ldg(a.tb), tlast = __ldg(a.tb + a.U);
  const int U = a.U;
  const size_t rowQ = (size_t)(U + 1);
  float acc[R];
#pragma unroll
  for (int i = 0; i < R; ++i) acc[i] = 0.f;
  const double dlane = (double)(x0 + lane), drow = (double)y0;
  for (int m = 0; m < a.cnt; ++m) {
    const size_t r = (size_t)z * a.cstride + m;
    const ViewGeom& G = a.vg[r];
    const bool xm = G.xmajor != 0;
    const float sgn = G.sgn;
    const double2* fcr = a.fc + r * rowQ;
    const Cell* qrow = reinterpret_cast<const Cell*>(a.sq) + r * rowQ;
    // first edge of this lane: x-major views: line li = x0 + lane, edge ck = y0;
    // y-major views: line li = y0, edge ck = x0 + lane
    double di = xm ? dlane : drow, dk = xm ? drow : dlane;
    int b;
    {
      const double ex = xm ? (dlane - a.ocx) * a.dx : (dlane - 0.5 - a.ocx) * a.dx;
      const double ey = xm ? (drow - 0.5 - a.ocy) * a.dx : (drow - a.ocy) * a.dx;
      const float vx = (float)(ex - G.sx), vy = (float)(ey - G.sy);
      const float cr = G.shx * vy - G.shy * vx, dt = G.shx * vx + G.shy * vy;
      const float t = a.dirt * __fdividef(cr, dt);
      if (!(t >= tfirst)) {
        b = 0;
      } else if (t >= tlast) {
        b = U - 1;
      } else {
        // a guess within a boundary or two; the walk below makes it exact
        const float mf = fminf(fmaxf((t - a.t0) * a.invdt, 0.f), (float)(a.M - 1));
        b = s_lut[(int)mf];
      }
    }
    const double s = (double)sgn;
    auto line_at = [&](int bb) {  // s-scaled boundary line (slope, offset)
      const double2 f = __ldg(fcr + bb);
      return make_double2(s * f.x, s * f.y);
    };
    dk *= s;
    double2 f0 = line_at(b), f1 = line_at(b + 1);
    double c0 = fma(di, f0.x, f0.y), c1 = fma(di, f1.x, f1.y);
    // Q at the current edge after moving the bracket onto it
    // (each loop moves b towards one end of [0, U - 1] and stops there)
    auto sample = [&]() {
      while (b < U - 1 && dk >= c1) {
        ++b;
        f0 = f1;
        c0 = c1;
        f1 = line_at(b + 1);
        c1 = fma(di, f1.x, f1.y);
      }
      while (b > 0 && dk < c0) {
        --b;
        f1 = f0;
        c1 = c0;
        f0 = line_at(b);
        c0 = fma(di, f0.x, f0.y);
      }
      const float frac = fminf(fmaxf((float)(dk - c0) * rcp_approx((float)(c1 - c0)), 0.f), 1.f);
      PhiS<M> q;
      q.load(qrow + b, frac);
      return q;
    };
    if (xm) {
      // the lane's column; the edge moves one row per step
      PhiS<M> prev = sample();
#pragma unroll
      for (int i = 0; i < R; ++i) {
        dk += s;
        const PhiS<M> cur = sample();
        acc[i] = fmaf(sgn, cur.diff(prev), acc[i]);
        prev = cur;
      }
    } else {
      // the lane's column edge; the line moves one row per step
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (i) {
          di += 1.0;
          c0 += f0.x;
          c1 += f1.x;
        }
        const PhiS<M> cur = sample();
        const PhiS<M> nxt = cur.down();
        acc[i] = fmaf(sgn, nxt.diff(cur), acc[i]);
      }
    }
  }
  const int ix = x0 + lane;
  if (lane >= PX || ix >= a.XN) return;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int iy = y0 + i;
    if (iy >= a.YN) break;
    const size_t pix = (size_t)iy * a.XN + ix;
    const size_t idx = (size_t)z * a.XN * a.YN + pix;
    const float mk = a.mask ? (float)a.mask[pix] : 1.f;
    float val = acc[i] * mk;
    if (a.x) {
      const float cs = __ldg(a.colsum + pix);
      const float t = cs != 0.f ? __fdiv_rn(val, cs) : val;
      val = a.x[idx] + t;
      if (a.nonneg) val = fmaxf(val, 0.f);
      a.x[idx] = val;
    } else {
      a.out[idx] = val;
    }
  }
}

// The reference backprojector's formula (AAPM_script/MultiSlicesBackGPU.cu:115-184,
// as k_back_ref) per slice: voxel-driven, angular detector coordinate
// alpha = asin(cross / (|s| l)) (here as the equal atan(cross / dot), in
// FP64), footprint half-width dx ddv / (2 l^2) and weight dx l / ddv (FP32,
// relative terms), coordinate alpha / dbeta + detCntIdx + 1 in FP64 per
// (voxel, view), then the two samples of the channel prefix sums in table
// precision.  Warp = 32 consecutive pixels of a row x R rows of one slice;
// the OS-SART update (or the plain backprojection) is fused as in
// k_ps_back_adj, with k_back_ref's mask rule (masked voxels get 0).
template <int M>
__global__ void __launch_bounds__(256) k_ps_back_ref(PsBackArgs a) {
  constexpr int R = kPsRefRows, PX = 32;
  using Cell = typename PsCell<M>::T;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int z = blockIdx.z;
  const int x0 = (blockIdx.x * 2 + (w & 1)) * PX, y0 = (blockIdx.y * 4 + (w >> 1)) * R;
  if (x0 >= a.XN || y0 >= a.YN) return;  // uniform per warp
  const int ix = x0 + lane;
  const int U = a.U;
  const double Ud = (double)U;
  const size_t rowQ = (size_t)(U + 1);
  const float dxf = (float)a.dx, hdx = (float)(a.dx * 0.5);
#if DDFAN_PS_REF_FIXED
  const double two32 = 4294967296.0;
  const double K32 = a.inv_dbeta * two32, C32 = a.cnt_ref * two32;  // coordinate per radian, offset; x 2^32
  const float hdxK = (float)(a.dx * 0.5 * a.inv_dbeta * two32);
  const long long cmax = (long long)U << 32;
#endif
  float acc[R];
#pragma unroll
  for (int i = 0; i < R; ++i) acc[i] = 0.f;
  for (int m = 0; m < a.cnt; ++m) {
    const size_t r = (size_t)z * a.cstride + m;
    const double sx = a.vg[r].sx, sy = a.vg[r].sy;
    const bool xdom = fabs(sx) > fabs(sy);
    const Cell* qrow = reinterpret_cast<const Cell*>(a.sq) + r * rowQ;
    const double ddx = ((double)ix - a.ocx) * a.dx - sx;
    double alpha = 0.0, ddy_prev = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const double ddy = ((double)(y0 + i) - a.ocy) * a.dx - sy;
      // alpha = asin((s_y d_x - s_x d_y) / (|s| l)) is the signed angle from
      // -s to d: atan of the cross over the dot product (dot > 0 for voxels in
      // front of the source), which needs no square root in FP64.  Down the
      // column the angle moves by the angle from the previous row's d to this
      // one, whose tangent t = d_x (dy_i - dy_{i-1}) / (d_{i-1} . d_i) is exact
      // and small; for |t| <= 0.05 the series t - t^3/3 + t^5/5 - t^7/7 is
      // exact to FP64 rounding (next term below 2e-13 t), otherwise the full
      // atan.  The half-width and the weight only need FP32.
      bool full = i == 0;
      if (!full) {
#if DDFAN_PS_REF_NEWTON
        // 1 / (d_{i-1} . d_i) from the FP32 approximate reciprocal (relative
        // error below 2^-22) and one FP64 Newton step (error squared: ~1e-13)
        const double den = fma(ddy_prev, ddy, ddx * ddx);
        const double r0 = (double)rcp_approx((float)den);
        const double rr = r0 * fma(-den, r0, 2.0);
        const double t = ddx * (ddy - ddy_prev) * rr;
#else
        const double t = ddx * (ddy - ddy_prev) / fma(ddy_prev, ddy, ddx * ddx);
#endif
        if (fabs(t) <= 0.05) {
          const double t2 = t * t;
          alpha += t * fma(t2, fma(t2, fma(t2, -1.0 / 7.0, 1.0 / 5.0), -1.0 / 3.0), 1.0);
        } else {
          full = true;
        }
      }
      if (full) alpha = atan((sy * ddx - sx * ddy) / -(sx * ddx + sy * ddy));
      ddy_prev = ddy;
      const float fx = (float)ddx, fy = (float)ddy, fdv = xdom ? fx : fy;
      const float l2 = fmaf(fx, fx, fy * fy);
      const double da = (double)(__fdividef(fdv, l2) * hdx);
      const float wt = __fdividef(dxf, fdv) * sqrtf(l2);
#if DDFAN_PS_REF_FIXED
      // both channel coordinates in 32.32 fixed point: the centre from FP64,
      // the half-width from FP32 (below a few channels, so its FP32 rounding
      // is ~1e-7 channel), clamped to [0, U] as integers; the fraction comes
      // from the low word (cell U holds the total with value 0, so a
      // coordinate of U samples it with fraction 0)
      (void)da;
      (void)Ud;
      const long long cc = __double2ll_rn(fma(alpha, K32, C32));
      // (bounded before the sums: a conversion out of range saturates)
      const long long hw = min(max(__float2ll_rn(__fdividef(fdv, l2) * hdxK), -(1LL << 50)), 1LL << 50);
      const long long cl = min(max(cc - hw, 0LL), cmax), cr = min(max(cc + hw, 0LL), cmax);
      const int iL = (int)(cl >> 32), iR = (int)(cr >> 32);
      PhiS<M> pL, pR;
      pL.load(qrow + iL, __int_as_float(0x3f800000 | ((unsigned)cl >> 9)) - 1.f);
      pR.load(qrow + iR, __int_as_float(0x3f800000 | ((unsigned)cr >> 9)) - 1.f);
#else
      const double cL = fmin(fmax((alpha - da) * a.inv_dbeta + a.cnt_ref, 0.0), Ud);
      const double cR = fmin(fmax((alpha + da) * a.inv_dbeta + a.cnt_ref, 0.0), Ud);
      const int iL = min((int)cL, U - 1), iR = min((int)cR, U - 1);
      PhiS<M> pL, pR;
      pL.load(qrow + iL, (float)(cL - iL));
      pR.load(qrow + iR, (float)(cR - iR));
#endif
      acc[i] = fmaf(pR.diff(pL), wt, acc[i]);
    }
  }
  if (ix >= a.XN) return;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int iy = y0 + i;
    if (iy >= a.YN) break;
    const size_t pix = (size_t)iy * a.XN + ix;
    const size_t idx = (size_t)z * a.XN * a.YN + pix;
    float val = (!a.mask || a.mask[pix] != 0) ? acc[i] : 0.f;
    if (a.x) {
      const float cs = __ldg(a.colsum + pix);
      const float t = cs != 0.f ? __fdiv_rn(val, cs) : val;
      val = a.x[idx] + t;
      if (a.nonneg) val = fmaxf(val, 0.f);
      a.x[idx] = val;
    } else {
      a.out[idx] = val;
    }
  }
}

}  // namespace ddfan
