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

// Prefix sums along every line: one CTA per (line, 32-slice tile), 256 threads.
// Thread (zl = tid % 8, kc = tid / 8) owns 4 slices and the chunk
// [kc*C, kc*C + C) of the line.  Chunk sums are combined by a warp-shuffle
// scan across the 4 chunk groups of a warp, then across the 8 warps through
// shared memory; every thread then writes its chunk's cells.  The inputs stay
// in registers between the two phases, so each value is read once.
// Writes Nw >= N cells per line (cells past the last value hold the total).
template <int M, int C>
__global__ void __launch_bounds__(256) k_sat(SatSrc s, float4* __restrict__ out, int nlines0,
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
  const int zb = blockIdx.y * 8 + zl;
  const bool zok = zb < ZB;
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
  __shared__ Acc4<M> wtot[8][8];
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
      run.store(out + (((size_t)line * Nw + k) * ZB + zb) * F4, v[j]);
      run.add(v[j]);
    }
  }
}

// ============================================================ forward projector

struct FwdArgs {
  const float4* satx;  // image rows table  [YN][XN][ZB]
  const float4* saty;  // image columns table [XN][YN][ZB]
  const ViewGeom* vg;
  const double2* fc;   // [PN][U+1]
  const float* cvd;    // [PN][U]
  const int* order;    // CTA row -> view (null = identity)
  float* out;          // [PN][U][Z]
  int PN, U, Z, ZB, XN, YN;
  float dx;
  int zlo, zhi;
};

// Branchless DD forward projection (AAPM_script/MultiSlicesProjGPU.cu:100-200)
// with exact interpolation weights.  Thread = CG consecutive channels x 4
// slices of one view; for every line ii it samples the U+1 shared boundary
// rays once each (channel u uses boundaries u and u+1) and adds
// (Phi(c_{u+1}) - Phi(c_u)) / len_u, len_u the footprint length in mm.
template <int M, int ZL, int CG>
__global__ void __launch_bounds__(128) k_fwd(FwdArgs a) {
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NG = 32 / ZL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int zl = lane % ZL, g = lane / ZL;
  const int p = a.order ? a.order[blockIdx.y] : blockIdx.y;
  const int zb = blockIdx.z * ZL + zl;
  const int u0 = ((blockIdx.x * 4 + w) * NG + g) * CG;
  if (u0 >= a.U || zb >= a.ZB) return;  // no block-level synchronisation below
  const bool xm = a.vg[p].xmajor != 0;
  const int nl = xm ? a.XN : a.YN, N = xm ? a.YN : a.XN;
  const float4* sat = xm ? a.saty : a.satx;
  const size_t rowstride = (size_t)a.ZB * F4;  // one k step
  double F[CG + 1], Cc[CG + 1];
#pragma unroll
  for (int b = 0; b <= CG; ++b) {
    const int ub = min(u0 + b, a.U);
    const double2 t = a.fc[(size_t)p * (a.U + 1) + ub];
    F[b] = t.x;
    Cc[b] = t.y;
  }
  float acc[CG][4];
#pragma unroll
  for (int b = 0; b < CG; ++b) acc[b][0] = acc[b][1] = acc[b][2] = acc[b][3] = 0.f;
  const double Nd = (double)N;
  const float4* base = sat + (size_t)zb * F4;
  for (int ii = 0; ii < nl; ++ii) {
    const float4* line = base + (size_t)ii * N * rowstride;
    const double di = (double)ii;
    Phi4<M> prev;
    double cprev = 0.0;
#pragma unroll
    for (int b = 0; b <= CG; ++b) {
      const double c = fma(di, F[b], Cc[b]);
      const double cc = fmin(fmax(c, 0.0), Nd);
      const int i0 = min((int)cc, N - 1);
      const float f = (float)(cc - (double)i0);
      Phi4<M> ph;
      ph.load(line + (size_t)i0 * rowstride, f);
      if (b > 0) {
        const float inv = __frcp_rn((float)(c - cprev) * a.dx);
        float d[4];
        ph.diff(prev, d);
#pragma unroll
        for (int s = 0; s < 4; ++s) acc[b - 1][s] = fmaf(d[s], inv, acc[b - 1][s]);
      }
      prev = ph;
      cprev = c;
    }
  }
#pragma unroll
  for (int b = 0; b < CG; ++b) {
    const int u = u0 + b;
    if (u >= a.U) break;
    const float cv = __ldg(a.cvd + (size_t)p * a.U + u) * a.dx;
    float* o = a.out + ((size_t)p * a.U + u) * a.Z;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int z = zb * 4 + s;
      if (z >= a.zlo && z < a.zhi) o[z] = acc[b][s] * cv;
    }
  }
}

// ============================================================ backprojectors

struct BackEpi {
  float* out;            // [YN][XN][Z]
  const float* addend;   // added before the update (null = none)
  const float* xin;      // OS-SART: x_new = x_in + t / colSum (null = plain backprojection)
  const float* colsum;   // [YN][XN] column sums (slice 0), used with xin
  int nonneg;            // clamp the updated image at 0
  const uint8_t* mask;   // [YN][XN] or null
  int zlo, zhi;
};

__device__ __forceinline__ void back_store(const BackEpi& e, int ix, int iy, int zb, int XN, int Z,
                                           bool scale_by_mask, const float (&acc)[4]) {
  const size_t pix = (size_t)iy * XN + ix;
  const float m = e.mask ? (float)e.mask[pix] : 1.f;
  const float cs = e.xin ? __ldg(e.colsum + pix) : 0.f;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int z = zb * 4 + s;
    if (z < e.zlo || z >= e.zhi) continue;
    const size_t idx = pix * Z + z;
    float val = scale_by_mask ? acc[s] * m : (m != 0.f ? acc[s] : 0.f);
    if (e.addend) val += e.addend[idx];
    if (e.xin) {
      // x += t / colSum where colSum != 0, else x += t (AAPM_script/OSSART_AAPM.m:94-97)
      const float t = cs != 0.f ? __fdiv_rn(val, cs) : val;
      val = e.xin[idx] + t;
      if (e.nonneg) val = fmaxf(val, 0.f);
    }
    e.out[idx] = val;
  }
}

struct RefArgs {
  const float4* satq;   // sinogram table [PN][U+1][ZB]
  const ViewGeom* vg;
  int PN, U, Z, ZB, XN, YN;
  double ocx, ocy, dx, inv_sid, inv_dbeta, cnt;  // cnt = detCntIdx + 1 - 0.5
  BackEpi epi;
};

// Reference backprojector formula (AAPM_script/MultiSlicesBackGPU.cu:115-184):
// voxel-driven, angular detector coordinate alpha = asin(cross / (|s| l)),
// footprint half-width dx * ddv / (2 l^2), weight dx l / ddv, coordinate
// alpha / dbeta + detCntIdx + 1 -- all evaluated in double, then the two
// samples of the channel prefix-sum table are differenced in table precision.
// Thread = VG consecutive voxels along x of one row x 4 slices.
template <int M, int ZL, int VG>
__global__ void __launch_bounds__(128) k_back_ref(RefArgs a) {
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NG = 32 / ZL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int zl = lane % ZL, g = lane / ZL;
  const int zb = blockIdx.z * ZL + zl;
  const int nseg = (a.XN + VG - 1) / VG;
  const int seg = (blockIdx.x * 4 + w) * NG + g;
  if (seg >= nseg * a.YN || zb >= a.ZB) return;
  const int iy = seg / nseg, ix0 = (seg % nseg) * VG;
  const int nv = min(VG, a.XN - ix0);
  unsigned on = 0;
#pragma unroll
  for (int v = 0; v < VG; ++v)
    if (v < nv && (!a.epi.mask || a.epi.mask[(size_t)iy * a.XN + ix0 + v] != 0)) on |= 1u << v;
  float acc[VG][4];
#pragma unroll
  for (int v = 0; v < VG; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.f;
  const double vy = (iy - a.ocy) * a.dx;
  const double Ud = (double)a.U;
  const size_t rowstride = (size_t)a.ZB * F4;
  for (int p = 0; p < a.PN; ++p) {
    const double sx = a.vg[p].sx, sy = a.vg[p].sy;
    const bool selx = fabs(sx) > fabs(sy);
    const float4* base = a.satq + ((size_t)p * (a.U + 1) * a.ZB + zb) * F4;
#pragma unroll
    for (int v = 0; v < VG; ++v) {
      if (!(on >> v & 1u)) continue;
      const double vx = (ix0 + v - a.ocx) * a.dx;
      const double ddx = vx - sx, ddy = vy - sy;
      const double l2 = ddx * ddx + ddy * ddy;
      const double l = sqrt(l2);
      const double alpha = asin((sy * ddx - sx * ddy) * a.inv_sid / l);
      const double ddv = selx ? ddx : ddy;
      const double da = ddv / l2 * a.dx * 0.5;
      const float cosv = (float)(a.dx / ddv * l);
      const double cL = fmin(fmax((alpha - da) * a.inv_dbeta + a.cnt, 0.0), Ud);
      const double cR = fmin(fmax((alpha + da) * a.inv_dbeta + a.cnt, 0.0), Ud);
      const int iL = min((int)cL, a.U - 1), iR = min((int)cR, a.U - 1);
      Phi4<M> pL, pR;
      pL.load(base + (size_t)iL * rowstride, (float)(cL - iL));
      pR.load(base + (size_t)iR * rowstride, (float)(cR - iR));
      float d[4];
      pR.diff(pL, d);
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[v][s] = fmaf(d[s], cosv, acc[v][s]);
    }
  }
#pragma unroll
  for (int v = 0; v < VG; ++v)
    if (v < nv) back_store(a.epi, ix0 + v, iy, zb, a.XN, a.Z, false, acc[v]);
}

struct AdjArgs {
  const float4* satq;   // weighted sinogram table [PN][U+1][ZB], weight r_u / |dir_u.axis|
  const ViewGeom* vg;
  const double2* fc;    // [PN][U+1]
  const float* tb;      // fan tangents of the boundaries, increasing, U+1
  const uint16_t* lut;  // bracket lookup, M entries
  float t0, invdt, dirt;
  int M;
  int PN, U, Z, ZB, XN, YN;
  double ocx, ocy, dx;
  BackEpi epi;
};

// Exact transpose of k_fwd.  For a view integrated along lines ii, pixel k of
// line ii receives sum_u w_u * (fraction of footprint u inside [k, k+1]),
// w_u = r_u / |dir_u.axis| -- which is the difference of the channel prefix
// sum Q of w at the fractional boundary index beta of the pixel's two edges:
// beta(c) = b + (c - c_b(ii)) / (c_{b+1}(ii) - c_b(ii)) with the forward's own
// c_b(ii).  Thread = VG consecutive pixels along one line (so VG+1 edges)
// x 4 slices; XM selects the lines (x columns for xmajor views, y rows
// otherwise) and the kernel visits only the views of that orientation.
template <int M, int ZL, int VG, bool XM>
__global__ void __launch_bounds__(128) k_back_adj(AdjArgs a) {
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NG = 32 / ZL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int zl = lane % ZL, g = lane / ZL;
  const int zb = blockIdx.z * ZL + zl;
  const int nl = XM ? a.XN : a.YN, N = XM ? a.YN : a.XN;
  const int nseg = (N + VG - 1) / VG;
  const int seg = (blockIdx.x * 4 + w) * NG + g;
  if (seg >= nseg * nl || zb >= a.ZB) return;
  const int ii = seg / nseg, k0 = (seg % nseg) * VG;
  const int nv = min(VG, N - k0);
  float acc[VG][4];
#pragma unroll
  for (int v = 0; v < VG; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.f;
  const double lineX = (ii - (XM ? a.ocx : a.ocy)) * a.dx;  // world coordinate of the line
  const double ock = XM ? a.ocy : a.ocx;
  const double di = (double)ii;
  const size_t rowstride = (size_t)a.ZB * F4;
  const float tfirst = __ldg(a.tb), tlast = __ldg(a.tb + a.U);
  for (int p = 0; p < a.PN; ++p) {
    if ((a.vg[p].xmajor != 0) != XM) continue;
    const double sx = a.vg[p].sx, sy = a.vg[p].sy;
    const float shx = a.vg[p].shx, shy = a.vg[p].shy, sgn = a.vg[p].sgn;
    const float4* base = a.satq + ((size_t)p * (a.U + 1) * a.ZB + zb) * F4;
    const double2* fcp = a.fc + (size_t)p * (a.U + 1);
    Phi4<M> prev;
#pragma unroll
    for (int e = 0; e <= VG; ++e) {
      if (e > nv) break;
      const double ck = (double)(k0 + e);             // edge position (texel-sample coords)
      const double along = (ck - 0.5 - ock) * a.dx;   // its world coordinate along the line
      const float vx = (float)((XM ? lineX : along) - sx);
      const float vy = (float)((XM ? along : lineX) - sy);
      const float cr = shx * vy - shy * vx, dt = shx * vx + shy * vy;
      const float t = a.dirt * __fdividef(cr, dt);
      int b;
      float frac = 0.f;
      if (!(t >= tfirst)) {
        b = 0;
      } else if (t >= tlast) {
        b = a.U;
      } else {
        const int m = (int)fminf(fmaxf((t - a.t0) * a.invdt, 0.f), (float)(a.M - 1));
        b = __ldg(a.lut + m);
        int guard = 0;
        while (b < a.U - 1 && __ldg(a.tb + b + 1) <= t && guard++ < 64) ++b;
        while (b > 0 && __ldg(a.tb + b) > t && guard++ < 128) --b;
        const double2 f0 = __ldg(fcp + b), f1 = __ldg(fcp + b + 1);
        const double c0 = fma(di, f0.x, f0.y), c1 = fma(di, f1.x, f1.y);
        frac = __fdiv_rn((float)(ck - c0), (float)(c1 - c0));
        frac = fminf(fmaxf(frac, 0.f), 1.f);
      }
      Phi4<M> ph;
      ph.load(base + (size_t)b * rowstride, frac);
      if (e > 0) {
        float d[4];
        ph.diff(prev, d);
#pragma unroll
        for (int s = 0; s < 4; ++s) acc[e - 1][s] = fmaf(sgn, d[s], acc[e - 1][s]);
      }
      prev = ph;
    }
  }
#pragma unroll
  for (int v = 0; v < VG; ++v) {
    if (v >= nv) break;
    const int k = k0 + v;
    back_store(a.epi, XM ? ii : k, XM ? k : ii, zb, a.XN, a.Z, true, acc[v]);
  }
}

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

}  // namespace ddfan
