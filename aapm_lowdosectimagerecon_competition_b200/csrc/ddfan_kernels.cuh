// ddfan_kernels.cuh -- the sm_100a kernels of the fan-beam DD path.
//
// Thread layout shared by the projector kernels: a warp is NG = 32/ZL groups
// of ZL lanes; the ZL lanes of a group own consecutive 4-slice blocks (one
// float4 per lane per cell plane, so a group reads ZL*16 contiguous bytes per
// plane), the NG groups own different channels / voxels.  All slices of a
// call share the view angles, so every lane of a group walks the same
// geometry and the gathers of a group are contiguous in z.
#pragma once
#include "ddfan_device.cuh"

namespace ddfan {

// ============================================================ view geometry

struct GeomConsts {
  double x0, y0, dx, ocx, ocy;
  const double* bx;  // boundaries (U+1), float-rounded as the reference stores them
  const double* by;
  const double* xd;  // channel centres (U)
  const double* yd;
  double sh0x, sh0y;  // unit vector source -> rotation centre at angle 0
  int U, XN, YN;
};

// Wrap to [0, 2 pi) the way regularizeAngle does (AAPM_script/utilities.cuh:143-148).
__device__ inline double wrap_angle(double c) {
  const double TWOPI = 6.283185307179586;
  int guard = 0;
  while (c >= TWOPI && guard < 1 << 20) { c -= TWOPI; ++guard; }
  while (c < 0.0 && guard < 1 << 21) { c += TWOPI; ++guard; }
  return c;
}

// One CTA per view.  Writes, in double, the boundary lines of the forward
// kernel (AAPM_script/MultiSlicesProjGPU.cu:120-168) in texel-sample
// coordinates: along line ii the boundary ray b crosses the prefix-sum axis at
// c_b(ii) = ii * F_b + C_b (c = texture coordinate - 0.5), and the per-channel
// ray weight 1/|dir.axis| (the reference's constVal is dx times this).
static __global__ void k_view_geom(GeomConsts g, const float* __restrict__ angs, int angs_stride, int PN,
                            ViewGeom* __restrict__ vg, double2* __restrict__ fc,
                            float* __restrict__ cvd) {
  const int p = blockIdx.x;
  if (p >= PN) return;
  const double th = wrap_angle((double)angs[(size_t)p * angs_stride]);
  double sn, cs;
  sincos(th, &sn, &cs);
  const double sx = g.x0 * cs - g.y0 * sn, sy = g.x0 * sn + g.y0 * cs;
  const bool xm = fabs(cs) <= fabs(sn);
  const int U = g.U;
  auto line_of = [&](int b, double& F, double& C) {
    const double Bx = g.bx[b] * cs - g.by[b] * sn, By = g.bx[b] * sn + g.by[b] * cs;
    if (xm) {
      const double f = (By - sy) / (Bx - sx);
      F = f;
      C = ((-g.ocx * g.dx - Bx) * f + By) / g.dx + g.ocy + 0.5;
    } else {
      const double f = (Bx - sx) / (By - sy);
      F = f;
      C = ((-g.ocy * g.dx - By) * f + Bx) / g.dx + g.ocx + 0.5;
    }
  };
  for (int b = threadIdx.x; b <= U; b += blockDim.x) {
    double F, C;
    line_of(b, F, C);
    fc[(size_t)p * (U + 1) + b] = make_double2(F, C);
  }
  for (int u = threadIdx.x; u < U; u += blockDim.x) {
    const double Dx = g.xd[u] * cs - g.yd[u] * sn, Dy = g.xd[u] * sn + g.yd[u] * cs;
    const double ddx = Dx - sx, ddy = Dy - sy;
    const double nrm = sqrt(ddx * ddx + ddy * ddy);
    cvd[(size_t)p * U + u] = (float)(nrm / fabs(xm ? ddx : ddy));
  }
  if (threadIdx.x == 0) {
    double F0, C0, F1, C1;
    line_of(0, F0, C0);
    line_of(U, F1, C1);
    const double mid = 0.5 * ((xm ? g.XN : g.YN) - 1);
    const double d = (C1 - C0) + mid * (F1 - F0);
    ViewGeom v;
    v.cs = cs; v.sn = sn; v.sx = sx; v.sy = sy;
    v.shx = (float)(g.sh0x * cs - g.sh0y * sn);
    v.shy = (float)(g.sh0x * sn + g.sh0y * cs);
    v.sgn = d >= 0 ? 1.f : -1.f;
    v.xmajor = xm ? 1 : 0;
    vg[p] = v;
  }
}

// ============================================================ prefix-sum tables

// What a prefix-sum table is built from.
struct SatSrc {
  int kind;             // 0: image rows (line = y, k = x); 1: image columns (line = x, k = y); 2: sinogram
  const float* a;       // image [YN][XN][Z], or sinogram [lines][U][Z] (A x for the fused residual)
  const uint8_t* mask;  // image mask [YN][XN] or null
  const float* wgt;     // sinogram: per (line, channel) weight, or null (= 1)
  float wscale;         // sinogram: extra scale on the weight
  const float* y;       // fused OS-SART residual: measured sinogram [views][U][Z] or null
  const int* yview;     // line -> view index into y
  const float* rowsum;  // [lines][U] row sums (slice 0) of the subset
  int XN, YN, U, Z;
  int ZLt;              // z-blocks per z-tile of the output layout
  int zb0, zb1;         // z-blocks built: [zb0, zb1); grid y covers them 8 at a time
  // Per-slice view angles (solver): line = slot of the z-tile's view range
  // ztd[zt] = {first geometry row, count, -, -}; geometry row r is raw view
  // g = r / Mc + (r % Mc) * nOS; slice z reads its view g - soff[z] of y when
  // that lies in [0, T) (else the residual is 0), with row sum row
  // (view - ksub) / nOS.  Null ztd: lines are views (yview, rowsum by line).
  const int4* ztd;
  const int* soff;
  int Mc, nOS, ksub, T;
};

__device__ __forceinline__ void sat_load(const SatSrc& s, int line, int k, int zb,
                                         float (&v)[4]) {
  size_t base;
  float m = 1.f;
  if (s.kind == 0) {
    const size_t pix = (size_t)line * s.XN + k;
    base = pix * s.Z;
    if (s.mask) m = (float)s.mask[pix];
  } else if (s.kind == 1) {
    const size_t pix = (size_t)k * s.XN + line;
    base = pix * s.Z;
    if (s.mask) m = (float)s.mask[pix];
  } else {
    const size_t e = (size_t)line * s.U + k;
    base = e * s.Z;
    m = s.wgt ? __ldg(s.wgt + e) * s.wscale : s.wscale;
  }
  const int z0 = zb * 4;
  if (z0 >= s.Z) {  // padding block of the last z-tile
    v[0] = v[1] = v[2] = v[3] = 0.f;
    return;
  }
  if (s.kind == 2 && s.ztd) {
    const int4 d = s.ztd[zb / s.ZLt];
    if (line >= d.y) {
      v[0] = v[1] = v[2] = v[3] = 0.f;
      return;
    }
    const int r = d.x + line;
    const long long g = (long long)(r / s.Mc) + (long long)(r % s.Mc) * s.nOS;
    const float mw = s.wgt ? __ldg(s.wgt + (size_t)r * s.U + k) * s.wscale : s.wscale;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int z = z0 + i;
      float val = 0.f;
      if (z < s.Z) {
        const long long ib = g - (long long)__ldg(s.soff + z);
        if (ib >= 0 && ib < s.T) {
          const float ax = __ldg(s.a + base + z);
          const float rs = __ldg(s.rowsum + (size_t)((ib - s.ksub) / s.nOS) * s.U + k);
          const float yv = __ldg(s.y + ((size_t)ib * s.U + k) * s.Z + z);
          // (y - A x) / rowSum where rowSum != 0, else A x (AAPM_script/OSSART_AAPM.m:88)
          val = rs != 0.f ? __fdiv_rn(__fsub_rn(yv, ax), rs) : ax;
        }
      }
      v[i] = val * mw;
    }
    return;
  }
  if ((s.Z & 3) == 0) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(s.a + base + z0));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = (z0 + i < s.Z) ? __ldg(s.a + base + z0 + i) : 0.f;
  }
  if (s.kind == 2 && s.y) {
    // r = (y - A x) / rowSum where rowSum != 0, else A x (AAPM_script/OSSART_AAPM.m:88)
    const float rs = __ldg(s.rowsum + (size_t)line * s.U + k);
    const size_t yb = ((size_t)__ldg(s.yview + line) * s.U + k) * s.Z + z0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (z0 + i < s.Z && rs != 0.f) v[i] = __fdiv_rn(__fsub_rn(__ldg(s.y + yb + i), v[i]), rs);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] *= m;
}

// Prefix sums along every line: one CTA per (line, 32-slice tile), 512 threads.
// Thread (zl = tid % 8, kc = tid / 8) owns 4 slices and the chunk
// [kc*C, kc*C + C) of the line (64 chunks).  Chunk sums are combined by a
// warp-shuffle scan across the 4 chunk groups of a warp, then across the 16
// warps through shared memory; every thread then writes its chunk's cells.
// The inputs stay in registers between the two phases, so each value is read
// once.
// Writes Nw >= N cells per line (cells past the last value hold the total).
template <int M, int C>
__global__ void __launch_bounds__(512) k_sat(SatSrc s, float4* __restrict__ out, int nlines0,
                                             int nlines1, float4* __restrict__ out1, int N0,
                                             int N1, int Nw0, int Nw1, int ZB) {
  constexpr int F4 = CellInfo<M>::F4;
  const int which = blockIdx.z;  // 0 or 1: two tables in one launch (image rows / columns)
  const int line = blockIdx.x;
  const int nlines = which ? nlines1 : nlines0;
  if (line >= nlines) return;  // uniform per CTA
  if (which) { s.kind = 1; out = out1; }
  const int N = which ? N1 : N0, Nw = which ? Nw1 : Nw0;
  const int zl = threadIdx.x & 7, kc = threadIdx.x >> 3;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int zb = s.zb0 + blockIdx.y * 8 + zl;
  const bool zok = zb < s.zb1 && zb < ZB;
  const int k0 = kc * C;
  float v[C][4];
  Acc4<M> acc;
  acc.zero();
#pragma unroll
  for (int j = 0; j < C; ++j) {
    const int k = k0 + j;
    if (zok && k < N) sat_load(s, line, k, zb, v[j]);
    else v[j][0] = v[j][1] = v[j][2] = v[j][3] = 0.f;
    acc.add(v[j]);
  }
  Acc4<M> inc = acc;
#pragma unroll
  for (int off = 8; off <= 16; off <<= 1) {
    Acc4<M> o = inc.shfl_up(off);
    if (lane >= off) inc.add(o);
  }
  Acc4<M> exc = inc.shfl_up(8);
  if (lane < 8) exc.zero();
  __shared__ Acc4<M> wtot[16][8];  // [warp][z lane]: up to 512 threads
  if (lane >= 24) wtot[w][zl] = inc;
  __syncthreads();
  Acc4<M> run;
  run.zero();
  for (int w2 = 0; w2 < w; ++w2) run.add(wtot[w2][zl]);
  run.add(exc);
  if (!zok) return;
#pragma unroll
  for (int j = 0; j < C; ++j) {
    const int k = k0 + j;
    if (k < Nw) {
      const int zt = zb / s.ZLt;
      run.store(out + (((size_t)line * Nw + k) * ZB + (size_t)zt * s.ZLt) * F4 + (zb - zt * s.ZLt), s.ZLt,
                v[j]);
      run.add(v[j]);
    }
  }
}

}  // namespace ddfan

#include "ddfan_proj_kernels.cuh"
#include "ddfan_dd_kernels.cuh"

namespace ddfan {

// ============================================================ OS-SART helpers

// FISTA momentum after an iteration (AAPM_script/OSSART_AAPM.m:111-115):
// t1 = (1 + sqrt(1 + 4 t0^2)) / 2, x += (t0 - 1) / t1 (x - x_prev); the
// result is also the next iteration's x_prev.  t0 lives on the device so the
// step can sit in a CUDA graph; k_fista_t advances it afterwards.
static __global__ void k_fista(float* __restrict__ x, float* __restrict__ xprev, size_t n,
                        const double* __restrict__ t0p) {
  const double t0 = *t0p;
  const double t1 = (1.0 + sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;
  const float mom = (float)((t0 - 1.0) / t1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float xv = x[i];
    const float v = xv + mom * (xv - xprev[i]);
    x[i] = v;
    xprev[i] = v;
  }
}

static __global__ void k_fista_t(double* t0p) {
  const double t0 = *t0p;
  *t0p = (1.0 + sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;
}

// The same for many solves in one launch pair: blockIdx.y is the solve.
struct FistaDesc {
  float* x;
  float* xprev;
  size_t n;
  double* t;
};

static __global__ void k_fista_batch(const FistaDesc* __restrict__ d) {
  const FistaDesc f = d[blockIdx.y];
  const double t0 = *f.t;
  const double t1 = (1.0 + sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;
  const float mom = (float)((t0 - 1.0) / t1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < f.n; i += (size_t)gridDim.x * blockDim.x) {
    const float xv = f.x[i];
    const float v = xv + mom * (xv - f.xprev[i]);
    f.x[i] = v;
    f.xprev[i] = v;
  }
}

static __global__ void k_fista_t_batch(const FistaDesc* __restrict__ d, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double* tp = d[i].t;
    const double t0 = *tp;
    *tp = (1.0 + sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;
  }
}

}  // namespace ddfan
