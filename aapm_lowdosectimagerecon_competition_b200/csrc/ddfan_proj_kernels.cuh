// ddfan_proj_kernels.cuh -- forward projector and the two backprojectors.
//
// All three kernels split their work the same way.  The geometry of a sample
// (which prefix-sum cell, which interpolation fraction, which weight) depends
// on the view and on the position in the image plane but not on the slice, so
// a CTA first computes it ONCE for its whole tile into shared memory (phase G,
// FP64 where the reference formula needs it), then every (channel-or-voxel
// group, z-lane) thread streams the cells of its 4 slices through it
// (phase A).  A group is ZL consecutive lanes owning consecutive 4-slice
// blocks, so each gather of a group is ZL * 48 contiguous bytes.
#pragma once
#include "ddfan_device.cuh"

// Resident CTAs per SM the register allocation is sized for (256 threads each:
// 4 -> at most 64 registers per thread, 2 -> 128).  Measured choices (96-view
// c3 subset); overridable at build time for tuning sweeps.  The forward
// projector with hi/lo cells runs faster with 2 CTAs and 128 registers, which
// keep four lines of gathers in flight (3.69 -> 3.54 ms); with FP32 or FP64
// cells, or narrower z-tiles, 4 CTAs stay faster.
#ifndef DDFAN_FWD_MIN_CTAS
#define DDFAN_FWD_MIN_CTAS 4
#endif
#ifndef DDFAN_FWD_MIN_CTAS_WIDE
#define DDFAN_FWD_MIN_CTAS_WIDE 2
#endif
#ifndef DDFAN_REF_MIN_CTAS
#define DDFAN_REF_MIN_CTAS 3
#endif
#ifndef DDFAN_ADJ_MIN_CTAS
#define DDFAN_ADJ_MIN_CTAS 4
#endif
// lines of a forward chunk unrolled together (more gathers in flight per thread)
#ifndef DDFAN_FWD_LINE_UNROLL
#define DDFAN_FWD_LINE_UNROLL 1
#endif
#ifndef DDFAN_FWD_LINE_UNROLL_WIDE
#define DDFAN_FWD_LINE_UNROLL_WIDE 4
#endif

namespace ddfan {

// per cell format M and z-tile width ZL: the wide setting only pays for hi/lo
// cells on 8-block tiles (with 4 blocks, as per-slice-angle solves use, it
// cost 10 %; with FP64 cells, whose double sums need more registers, 45 %)
template <int M, int ZL> struct FwdTuning {
  static constexpr bool wide = M == SAT_HILO && ZL == 8;
  static constexpr int min_ctas = wide ? DDFAN_FWD_MIN_CTAS_WIDE : DDFAN_FWD_MIN_CTAS;
  static constexpr int line_unroll = wide ? DDFAN_FWD_LINE_UNROLL_WIDE : DDFAN_FWD_LINE_UNROLL;
};

// Stable partition of a call's views, x-major views first:
// order[0, nx) are the x-major views, order[nx, PN) the others; counts = {nx, PN - nx}.
// One CTA of 1024 threads.
static __global__ void __launch_bounds__(1024) k_view_order(const ViewGeom* __restrict__ vg, int PN,
                                                            int* __restrict__ order,
                                                            int* __restrict__ counts) {
  __shared__ int sx[1024], sy[1024], tot;
  const int t = threadIdx.x, T = blockDim.x;
  const int ch = (PN + T - 1) / T;
  const int a = min(PN, t * ch), b = min(PN, a + ch);
  int nx = 0;
  for (int p = a; p < b; ++p) nx += vg[p].xmajor != 0;
  sx[t] = nx;
  sy[t] = (b - a) - nx;
  __syncthreads();
  if (t == 0) {
    int ax = 0, ay = 0;
    for (int i = 0; i < T; ++i) {
      const int u = sx[i], v = sy[i];
      sx[i] = ax;
      sy[i] = ay;
      ax += u;
      ay += v;
    }
    tot = ax;
    counts[0] = ax;
    counts[1] = ay;
  }
  __syncthreads();
  int ox = sx[t], oy = tot + sy[t];
  for (int p = a; p < b; ++p) {
    if (vg[p].xmajor) order[ox++] = p;
    else order[oy++] = p;
  }
}

// The same partition for many view ranges at once (one CTA per range):
// range r covers geometry rows [d.x, d.x + d.y); its slots 0..d.y-1 go to
// order[d.z ...], x-major first, and d.w receives the x-major count.
static __global__ void __launch_bounds__(1024) k_view_order_ranges(const ViewGeom* __restrict__ vg,
                                                                   int4* __restrict__ desc,
                                                                   int* __restrict__ order) {
  __shared__ int sx[1024], sy[1024], tot;
  const int4 d = desc[blockIdx.x];
  const ViewGeom* v = vg + d.x;
  int* o = order + d.z;
  const int PN = d.y;
  const int t = threadIdx.x, T = blockDim.x;
  const int ch = (PN + T - 1) / T;
  const int a = min(PN, t * ch), b = min(PN, a + ch);
  int nx = 0;
  for (int p = a; p < b; ++p) nx += v[p].xmajor != 0;
  sx[t] = nx;
  sy[t] = (b - a) - nx;
  __syncthreads();
  if (t == 0) {
    int ax = 0, ay = 0;
    for (int i = 0; i < T; ++i) {
      const int u = sx[i], w = sy[i];
      sx[i] = ax;
      sy[i] = ay;
      ax += u;
      ay += w;
    }
    tot = ax;
    desc[blockIdx.x].w = ax;
  }
  __syncthreads();
  int ox = sx[t], oy = tot + sy[t];
  for (int p = a; p < b; ++p) {
    if (v[p].xmajor) o[ox++] = p;
    else o[oy++] = p;
  }
}

// Per z-tile view ranges (solver with per-slice view angles): tile zt
// projects the views {x: first geometry row, y: count, z: offset of its slot
// order, w: x-major count}; output rows and sinogram-table rows are the
// tile's slots 0..count-1.  Null: every tile uses all PN views (rows = slots).
struct ZtRange {
  int gbase, count, ooff, nx;
};

__device__ __forceinline__ ZtRange zt_range(const int4* ztd, int zt, int PN, const int* counts) {
  ZtRange r;
  if (ztd) {
    const int4 d = ztd[zt];
    r.gbase = d.x; r.count = d.y; r.ooff = d.z; r.nx = d.w;
  } else {
    r.gbase = 0; r.count = PN; r.ooff = 0; r.nx = counts ? counts[0] : 0;
  }
  return r;
}

// ============================================================ forward projector

struct FwdArgs {
  const float4* satx;  // image rows table    [YN][XN][ZB]
  const float4* saty;  // image columns table [XN][YN][ZB]
  const ViewGeom* vg;
  const double2* fc;   // [PN][U+1] boundary lines c_b(ii) = ii * F + C
  const float* cvd;    // [PN][U]   1 / |dir.axis|
  const int* order;    // CTA row -> view (views of one orientation adjacent); null = identity
  float* out;          // [PN][U][Z]
  int PN, U, Z, ZB, XN, YN;
  float dx;
  int zlo, zhi;        // slices written
  int zt0;             // z-tile of grid z-index 0 (the grid covers the tiles of [zlo, zhi))
  const int4* ztd;     // per z-tile view ranges, or null
  int row0;            // CTA row of grid y-index 0 (views beyond 65535 go in further launches)
};

template <int ZL, int CG>
struct FwdTile {
  static constexpr int NT = 256;           // threads
  static constexpr int NG = NT / ZL;       // channel groups
  static constexpr int CW = NG * CG;       // channels per CTA
  static constexpr int NB = CW + 1;        // boundaries per CTA
  static constexpr int CC = 2048 / CW;     // lines per geometry chunk
};

// Branchless DD forward projection (AAPM_script/MultiSlicesProjGPU.cu:100-200)
// with exact interpolation weights.  CTA = one view x CW consecutive channels
// x 4*ZL slices.  Phase G: for CC lines at a time, the CW+1 boundary rays'
// cell index, fraction and every channel's 1/(footprint length) -- from the
// FP64 boundary lines.  Phase A: a thread owns CG consecutive channels x 4
// slices; channel u adds (Phi(c_{u+1}) - Phi(c_u)) / len_u on every line.
template <int M, int ZL, int CG>
__global__ void __launch_bounds__(256, FwdTuning<M, ZL>::min_ctas) k_fwd(FwdArgs a) {
  using T = FwdTile<ZL, CG>;
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NT = T::NT, CW = T::CW, NB = T::NB, CC = T::CC;
  __shared__ double2 s_fc[NB];
  __shared__ int2 s_geo[CC][NB];   // (cell index, fraction bits)
  __shared__ float s_inv[CC][CW];  // 1 / (footprint length in mm)
  const int tid = threadIdx.x;
  const int zl = tid % ZL, g = tid / ZL;
  const int zt = blockIdx.z + a.zt0;
  const ZtRange rg = zt_range(a.ztd, zt, a.PN, nullptr);
  const int row = a.row0 + (int)blockIdx.y;
  if (row >= rg.count) return;  // uniform per CTA
  const int slot = a.order ? a.order[rg.ooff + row] : row;
  const int p = rg.gbase + slot;  // geometry row
  const int zb = zt * ZL + zl;
  const int ub0 = blockIdx.x * CW;
  const bool xm = a.vg[p].xmajor != 0;
  const int nl = xm ? a.XN : a.YN, N = xm ? a.YN : a.XN;
  const float4* sat = xm ? a.saty : a.satx;
  const size_t rowstride = (size_t)a.ZB * F4;
  for (int b = tid; b < NB; b += NT) s_fc[b] = a.fc[(size_t)p * (a.U + 1) + min(ub0 + b, a.U)];
  const bool active = (ub0 + g * CG < a.U) && (zb < a.ZB);
  // plane 0 of this lane's block in row 0 (see the table layout in ddfan_device.cuh)
  const float4* base = sat + (size_t)(active ? zt * ZL : 0) * F4 + zl;
  // ray sums: each chunk of CC lines is summed into a fresh FP32 partial that
  // is then added to the total, so a 512-line sum rounds like ~sqrt(512/CC)
  // terms instead of 512
  float acc[CG][4];
#pragma unroll
  for (int j = 0; j < CG; ++j)
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[j][s] = 0.f;
  const double Nd = (double)N;
  const float dx = a.dx;
  __syncthreads();
  for (int ii0 = 0; ii0 < nl; ii0 += CC) {
    for (int e = tid; e < CC * NB; e += NT) {
      const int col = e / NB, bb = e - col * NB;
      const double di = (double)(ii0 + col);
      const double2 f0 = s_fc[bb];
      const double c = fma(di, f0.x, f0.y);
      const double cc = fmin(fmax(c, 0.0), Nd);
      const int i0 = min((int)cc, N - 1);
      s_geo[col][bb] = make_int2(i0, __float_as_int((float)(cc - (double)i0)));
      if (bb < CW) {
        const double2 f1 = s_fc[bb + 1];
        s_inv[col][bb] = __frcp_rn((float)(fma(di, f1.x, f1.y) - c) * dx);
      }
    }
    __syncthreads();
    if (active) {
      const int ncol = min(CC, nl - ii0);
      float part[CG][4];
#pragma unroll
      for (int j = 0; j < CG; ++j) part[j][0] = part[j][1] = part[j][2] = part[j][3] = 0.f;
#pragma unroll(FwdTuning<M, ZL>::line_unroll)
      for (int col = 0; col < ncol; ++col) {
        const float4* line = base + (size_t)(ii0 + col) * N * rowstride;
        Phi4<M> prev;
        {
          const int2 gi = s_geo[col][g * CG];
          prev.load(line + (size_t)gi.x * rowstride, ZL, __int_as_float(gi.y));
        }
#pragma unroll
        for (int j = 0; j < CG; ++j) {
          const int2 gi = s_geo[col][g * CG + j + 1];
          Phi4<M> cur;
          cur.load(line + (size_t)gi.x * rowstride, ZL, __int_as_float(gi.y));
          const float inv = s_inv[col][g * CG + j];
          float d[4];
          cur.diff(prev, d);
#pragma unroll
          for (int s = 0; s < 4; ++s) part[j][s] = fmaf(d[s], inv, part[j][s]);
          prev = cur;
        }
      }
#pragma unroll
      for (int j = 0; j < CG; ++j)
#pragma unroll
        for (int s = 0; s < 4; ++s) acc[j][s] += part[j][s];
    }
    __syncthreads();
  }
  if (!active) return;
#pragma unroll
  for (int j = 0; j < CG; ++j) {
    const int u = ub0 + g * CG + j;
    if (u >= a.U) break;
    const float cv = __ldg(a.cvd + (size_t)p * a.U + u) * dx;
    float* o = a.out + ((size_t)slot * a.U + u) * a.Z;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int z = zb * 4 + s;
      if (z >= a.zlo && z < a.zhi) o[z] = acc[j][s] * cv;
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

// Voxel tile shared by the backprojectors: NG = 256/ZL groups arranged as LT
// lines x SPL segments of VG consecutive voxels along the line.
template <int ZL>
struct BackTile {
  static constexpr int NT = 256;
  static constexpr int NG = NT / ZL;
  static constexpr int VG = 8;              // voxels per thread
  static constexpr int SPL = 8;             // segments per line
  static constexpr int KT = SPL * VG;       // voxels per line in the tile
  static constexpr int LT = NG / SPL;       // lines per tile
  static constexpr int NV = LT * KT;        // voxels per tile
  static constexpr int NE = LT * (KT + 1);  // pixel edges per tile (exact adjoint)
  // shared-memory layout of a line's edges: one pad slot after every VG edges,
  // so the VG-edge runs of adjacent groups start 72 bytes apart (no bank conflicts)
  static constexpr int LS = KT + KT / VG + 1;
  static constexpr int NES = LT * LS;
};

struct RefArgs {
  const float4* satq;   // sinogram table [PN][U+1][ZB]
  const ViewGeom* vg;
  int PN, U, Z, ZB, XN, YN;
  double ocx, ocy, dx, inv_sid, inv_dbeta, cnt;  // cnt = detCntIdx + 1 - 0.5
  BackEpi epi;
  int zt0;  // z-tile of grid z-index 0
  const int4* ztd;  // per z-tile view ranges, or null
};

// Reference backprojector formula (AAPM_script/MultiSlicesBackGPU.cu:115-184):
// voxel-driven; angular detector coordinate alpha = asin(cross / (|s| l)),
// footprint half-width dx ddv / (2 l^2), weight dx l / ddv, coordinate
// alpha / dbeta + detCntIdx + 1.  Phase G evaluates that in FP64 once per
// (voxel, view) of the tile; phase A differences the two samples of the
// channel prefix sums in table precision.  Lines are image rows (k = x).
template <int M, int ZL>
__global__ void __launch_bounds__(256, DDFAN_REF_MIN_CTAS) k_back_ref(RefArgs a) {
  using T = BackTile<ZL>;
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NT = T::NT, VG = T::VG, SPL = T::SPL, KT = T::KT, LT = T::LT, NV = T::NV;
  constexpr int VC = (2048 / NV) < 1 ? 1 : ((2048 / NV) > 4 ? 4 : 2048 / NV);  // views per chunk
  __shared__ int2 s_i[VC][NV];
  __shared__ float2 s_f[VC][NV];
  __shared__ float s_w[VC][NV];
  __shared__ int s_p[VC];
  const int tid = threadIdx.x;
  const int zl = tid % ZL, g = tid / ZL;
  const int zt = blockIdx.z + a.zt0;
  const int zb = zt * ZL + zl;
  const int ntx = (a.XN + KT - 1) / KT;
  const int ty = blockIdx.x / ntx, tx = blockIdx.x - ty * ntx;
  const int y0 = ty * LT, x0 = tx * KT;
  const int l = g / SPL, sg = g - l * SPL;
  const int iy = y0 + l, ixs = x0 + sg * VG;
  const bool active = zb < a.ZB && iy < a.YN && ixs < a.XN;
  const ZtRange rg = zt_range(a.ztd, zt, a.PN, nullptr);
  float acc[VG][4];
#pragma unroll
  for (int v = 0; v < VG; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.f;
  const double Ud = (double)a.U;
  const size_t rowstride = (size_t)a.ZB * F4;
  for (int v0 = 0; v0 < rg.count; v0 += VC) {
    const int nvc = min(VC, rg.count - v0);
    if (tid < VC) s_p[tid] = v0 + tid;
    for (int e = tid; e < VC * NV; e += NT) {
      const int vv = e / NV, r = e - vv * NV;
      const int ly = r / KT, lx = r - ly * KT;
      const int yy = y0 + ly, xx = x0 + lx;
      int2 ii = make_int2(0, 0);
      float2 ff = make_float2(0.f, 0.f);
      float w = 0.f;
      if (vv < nvc && yy < a.YN && xx < a.XN &&
          (!a.epi.mask || a.epi.mask[(size_t)yy * a.XN + xx] != 0)) {
        const ViewGeom& G = a.vg[rg.gbase + v0 + vv];
        const double sx = G.sx, sy = G.sy;
        const double ddx = (xx - a.ocx) * a.dx - sx, ddy = (yy - a.ocy) * a.dx - sy;
        const double l2 = ddx * ddx + ddy * ddy;
        const double ln = sqrt(l2);
        const double alpha = asin((sy * ddx - sx * ddy) * a.inv_sid / ln);
        const double ddv = fabs(sx) > fabs(sy) ? ddx : ddy;
        const double da = ddv / l2 * a.dx * 0.5;
        w = (float)(a.dx / ddv * ln);
        const double cL = fmin(fmax((alpha - da) * a.inv_dbeta + a.cnt, 0.0), Ud);
        const double cR = fmin(fmax((alpha + da) * a.inv_dbeta + a.cnt, 0.0), Ud);
        ii = make_int2(min((int)cL, a.U - 1), min((int)cR, a.U - 1));
        ff = make_float2((float)(cL - ii.x), (float)(cR - ii.y));
      }
      s_i[vv][r] = ii;
      s_f[vv][r] = ff;
      s_w[vv][r] = w;
    }
    __syncthreads();
    if (active) {
      for (int vv = 0; vv < nvc; ++vv) {
        const float4* base = a.satq + ((size_t)s_p[vv] * (a.U + 1) * a.ZB + (size_t)zt * ZL) * F4 + zl;
#pragma unroll
        for (int v = 0; v < VG; ++v) {
          const int r = l * KT + sg * VG + v;
          const int2 ii = s_i[vv][r];
          const float2 ff = s_f[vv][r];
          Phi4<M> pL, pR;
          pL.load(base + (size_t)ii.x * rowstride, ZL, ff.x);
          pR.load(base + (size_t)ii.y * rowstride, ZL, ff.y);
          float d[4];
          pR.diff(pL, d);
          const float w = s_w[vv][r];
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[v][s] = fmaf(d[s], w, acc[v][s]);
        }
      }
    }
    __syncthreads();
  }
  if (!active) return;
#pragma unroll
  for (int v = 0; v < VG; ++v)
    if (ixs + v < a.XN) back_store(a.epi, ixs + v, iy, zb, a.XN, a.Z, false, acc[v]);
}

struct AdjArgs {
  const float4* satq;   // weighted sinogram table [PN][U+1][ZB], weight r_u / |dir_u.axis|
  const ViewGeom* vg;
  const double2* fc;    // [PN][U+1]
  const float* tb;      // fan tangents of the boundaries, increasing, U+1
  const uint16_t* lut;  // bracket lookup, M entries
  const int* order;     // views, x-major first
  const int* counts;    // {number of x-major views, others}
  float t0, invdt, dirt;
  int M;
  int PN, U, Z, ZB, XN, YN;
  double ocx, ocy, dx;
  BackEpi epi;
  int zt0;  // z-tile of grid z-index 0
  const int4* ztd;  // per z-tile view ranges (order, counts then unused), or null
};

// Exact transpose of k_fwd.  For a view integrated along lines ii, pixel k of
// line ii receives sum_u w_u * (fraction of footprint u inside [k, k+1]),
// w_u = r_u / |dir_u.axis| -- the difference of the channel prefix sum Q of w
// at the fractional boundary index beta of the pixel's two edges,
// beta(c) = b + (c - c_b(ii)) / (c_{b+1}(ii) - c_b(ii)), c_b(ii) the
// forward's own boundary lines.  b comes from the edge's fan tangent (lookup
// table + one correction step), the fraction from the FP64 lines.  Phase G
// computes (b, fraction) once per (edge, view) of the tile; a thread owns VG
// consecutive pixels of a line (VG + 1 edges) x 4 slices.  XM selects the
// lines (x columns for x-major views, y rows otherwise) and the views.
template <int M, int ZL, bool XM>
__global__ void __launch_bounds__(256, DDFAN_ADJ_MIN_CTAS) k_back_adj(AdjArgs a) {
  using T = BackTile<ZL>;
  constexpr int F4 = CellInfo<M>::F4;
  constexpr int NT = T::NT, VG = T::VG, SPL = T::SPL, KT = T::KT, LT = T::LT, NE = T::NE;
  constexpr int LS = T::LS, NES = T::NES;
  constexpr int VC = (1024 / NE) < 1 ? 1 : ((1024 / NE) > 4 ? 4 : 1024 / NE);
  constexpr int TBMAX = 1024, LUTMAX = 4096;
  __shared__ int2 s_geo[VC][NES];  // edge k of line l at l * LS + k + k / VG
  __shared__ int s_p[VC];
  __shared__ float s_sgn[VC];
  __shared__ float s_tb[TBMAX];
  __shared__ uint16_t s_lut[LUTMAX];
  const int tid = threadIdx.x;
  const int zl = tid % ZL, g = tid / ZL;
  const int zt = blockIdx.z + a.zt0;
  const int zb = zt * ZL + zl;
  const int nl = XM ? a.XN : a.YN, N = XM ? a.YN : a.XN;
  const int ntk = (N + KT - 1) / KT;
  const int tl = blockIdx.x / ntk, tk = blockIdx.x - tl * ntk;
  const int l0 = tl * LT, k0 = tk * KT;
  const int l = g / SPL, sg = g - l * SPL;
  const int ii = l0 + l, ks = k0 + sg * VG;
  const bool active = zb < a.ZB && ii < nl && ks < N;
  for (int i = tid; i <= a.U; i += NT) s_tb[i] = a.tb[i];
  for (int i = tid; i < a.M; i += NT) s_lut[i] = a.lut[i];
  const ZtRange rg = zt_range(a.ztd, zt, a.PN, a.counts);
  const int* order = a.order + rg.ooff;
  const int nx = rg.nx;
  const int vbeg = XM ? 0 : nx, vend = XM ? nx : rg.count;
  float acc[VG][4];
#pragma unroll
  for (int v = 0; v < VG; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.f;
  const size_t rowstride = (size_t)a.ZB * F4;
  const double ocl = XM ? a.ocx : a.ocy, ock = XM ? a.ocy : a.ocx;
  __syncthreads();
  const float tfirst = s_tb[0], tlast = s_tb[a.U];
  for (int v0 = vbeg; v0 < vend; v0 += VC) {
    const int nvc = min(VC, vend - v0);
    if (tid < VC && tid < nvc) {
      const int p = order[v0 + tid];
      s_p[tid] = p;
      s_sgn[tid] = a.vg[rg.gbase + p].sgn;
    }
    for (int e = tid; e < VC * NE; e += NT) {
      const int vv = e / NE, r = e - vv * NE;
      const int le = r / (KT + 1), ke = r - le * (KT + 1);
      const int li = l0 + le, ck = k0 + ke;
      int b = 0;
      float frac = 0.f;
      if (vv < nvc && li < nl && ck <= N) {
        const int p = rg.gbase + order[v0 + vv];
        const ViewGeom& G = a.vg[p];
        const double lineX = (li - ocl) * a.dx, along = ((double)ck - 0.5 - ock) * a.dx;
        const float vx = (float)((XM ? lineX : along) - G.sx);
        const float vy = (float)((XM ? along : lineX) - G.sy);
        const float cr = G.shx * vy - G.shy * vx, dt = G.shx * vx + G.shy * vy;
        const float t = a.dirt * __fdividef(cr, dt);
        if (!(t >= tfirst)) {
          b = 0;
        } else if (t >= tlast) {
          b = a.U;
        } else {
          const int m = (int)fminf(fmaxf((t - a.t0) * a.invdt, 0.f), (float)(a.M - 1));
          b = s_lut[m];
          int guard = 0;
          while (b < a.U - 1 && s_tb[b + 1] <= t && guard++ < 64) ++b;
          while (b > 0 && s_tb[b] > t && guard++ < 128) --b;
          const double2* fcp = a.fc + (size_t)p * (a.U + 1);
          const double2 f0 = __ldg(fcp + b), f1 = __ldg(fcp + b + 1);
          const double di = (double)li;
          const double c0 = fma(di, f0.x, f0.y), c1 = fma(di, f1.x, f1.y);
          frac = __fdiv_rn((float)((double)ck - c0), (float)(c1 - c0));
          frac = fminf(fmaxf(frac, 0.f), 1.f);
        }
      }
      s_geo[vv][le * LS + ke + ke / VG] = make_int2(b, __float_as_int(frac));
    }
    __syncthreads();
    if (active) {
      for (int vv = 0; vv < nvc; ++vv) {
        const float4* base = a.satq + ((size_t)s_p[vv] * (a.U + 1) * a.ZB + (size_t)zt * ZL) * F4 + zl;
        const float sgn = s_sgn[vv];
        // edges sg*VG .. sg*VG + VG of line l (the last one sits after a pad slot)
        const int2* geo = &s_geo[vv][l * LS + sg * (VG + 1)];
        Phi4<M> prev;
        {
          const int2 gi = geo[0];
          prev.load(base + (size_t)gi.x * rowstride, ZL, __int_as_float(gi.y));
        }
#pragma unroll
        for (int v = 0; v < VG; ++v) {
          const int2 gi = geo[v + 1 == VG ? VG + 1 : v + 1];
          Phi4<M> cur;
          cur.load(base + (size_t)gi.x * rowstride, ZL, __int_as_float(gi.y));
          float d[4];
          cur.diff(prev, d);
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[v][s] = fmaf(sgn, d[s], acc[v][s]);
          prev = cur;
        }
      }
    }
    __syncthreads();
  }
  if (!active) return;
#pragma unroll
  for (int v = 0; v < VG; ++v) {
    const int k = ks + v;
    if (k >= N) break;
    back_store(a.epi, XM ? ii : k, XM ? k : ii, zb, a.XN, a.Z, true, acc[v]);
  }
}

}  // namespace ddfan
