// ddfan_dd_kernels.cuh -- projector kernels that read the values themselves
// instead of prefix-sum tables (DDFAN_SAT_DIRECT).
//
// Every sample of the branchless DD path is a difference of two linearly
// interpolated prefix sums, Phi(c1) - Phi(c0), with Phi(c) = S[k] + f v[k]
// (k = floor of the clamped c, f its fraction; AAPM_script/
// MultiSlicesProjGPU.cu:161-170, MultiSlicesBackGPU.cu:175-179).  The
// difference telescopes to the values between the two positions:
//   k1 == k0:  (f1 - f0) v[k0]
//   k1 >  k0:  (1 - f0) v[k0] + sum_{k0<k<k1} v[k] + f1 v[k1]
//   k1 <  k0:  -f0 v[k0] - sum_{k1<k<k0} v[k] + (f1 - 1) v[k1]
// -- the same number in exact arithmetic, with no cancellation in FP32 and
// without building or reading a table.  A DD footprint covers one to three
// values at the geometries this path serves (the axis is chosen so that a ray
// crosses at most one cell per line, and channel and pixel pitch are
// comparable), so a sample reads one float per slice plus the one it shares
// with its neighbour, where a 48-byte hi/lo cell read 12 bytes per slice per
// boundary.  Wider footprints walk more values (any width is correct).
//
// Layouts: the image [YN][XN][P4] float4 (4 slices per float4, P4 = padded
// slices / 4) is read straight, masked beforehand; the sinogram operands
// [slot][U + 1][P4] float4 hold the (weighted) residual with a zero guard
// channel U, so a walk that ends on the last boundary (index U, fraction 0)
// reads a zero.  Geometry phases (FP64 boundary lines, brackets, fractions)
// are those of the prefix-sum kernels; only the gather changes.
#pragma once
#include "ddfan_proj_kernels.cuh"

namespace ddfan {

// Resident CTAs per SM the register allocation is sized for (256 threads:
// 2 -> up to 128 registers, which the 4-z-tile accumulators need without
// spilling).  Build-time knobs for tuning sweeps, like the tile shapes below.
#ifndef DDFAN_DD_FWD_MIN_CTAS
#define DDFAN_DD_FWD_MIN_CTAS 2
#endif
#ifndef DDFAN_DD_BACK_MIN_CTAS
#define DDFAN_DD_BACK_MIN_CTAS 2
#endif
// With DDFAN_DD_MIN_CTAS_BY_NZ the kernels of fewer z-tiles per thread (fewer
// accumulators) are built for one (NZ = 2: 80 registers) or two (NZ = 1: 64)
// more resident CTAs.  On a c3 subset forced to NZ = 2 this took the forward
// from 2.84 to 2.28 ms and the REF backprojector from 2.03 to 1.80 (NZ = 1:
// 3.59 -> 3.00, 3.56 -> 2.82); the NZ = 4 kernels are unchanged.
#ifndef DDFAN_DD_MIN_CTAS_BY_NZ
#define DDFAN_DD_MIN_CTAS_BY_NZ 1
#endif
// Work-list kernels: argument block copied to registers (1) or read in place
// through the read-only path (0).  The copy spilled at the 80-register
// budget of 2 z-tiles per thread (68-104 bytes against 12-24 for the grid
// kernels); read in place, batched c4 went from 17.1 to 18.7 iterations/s.
#ifndef DDFAN_DD_BATCH_ARGS_COPY
#define DDFAN_DD_BATCH_ARGS_COPY 0
#endif
template <int NZ, int BASE>
struct DdMinCtas {
  static constexpr int v = DDFAN_DD_MIN_CTAS_BY_NZ ? (NZ >= 4 ? BASE : (NZ == 2 ? BASE + 1 : BASE + 2)) : BASE;
};

// a += w v on 4 slices, as two packed fma.rn.f32x2 (sm_100: two lanes of
// round-to-nearest FMA per instruction, the same results as four fmaf; half
// the FMA instructions took a c3 subset's forward from 2.50 to 2.41 ms).
// DDFAN_FFMA2=0 builds the scalar form.
#ifndef DDFAN_FFMA2
#define DDFAN_FFMA2 1
#endif
__device__ __forceinline__ void fma2(float& a0, float& a1, float w, float v0, float v1) {
  asm("{\n\t.reg .b64 ra, rv, rw;\n\t"
      "mov.b64 ra, {%0, %1};\n\t"
      "mov.b64 rv, {%2, %3};\n\t"
      "mov.b64 rw, {%4, %4};\n\t"
      "fma.rn.f32x2 ra, rw, rv, ra;\n\t"
      "mov.b64 {%0, %1}, ra;\n\t}"
      : "+f"(a0), "+f"(a1)
      : "f"(v0), "f"(v1), "f"(w));
}
__device__ __forceinline__ void fma4(float (&a)[4], float w, const float4& v) {
#if DDFAN_FFMA2
  fma2(a[0], a[1], w, v.x, v.y);
  fma2(a[2], a[3], w, v.z, v.w);
#else
  a[0] = fmaf(w, v.x, a[0]);
  a[1] = fmaf(w, v.y, a[1]);
  a[2] = fmaf(w, v.z, a[2]);
  a[3] = fmaf(w, v.w, a[3]);
#endif
}

// The walk from (k0, f0) to (k1, f1) as three weights: w0 on the value at
// k0, wm on the value one step on (an interior value when n = |k1 - k0| >= 2,
// else 0: that value is then the end value or past it), we on the value at k1
// (0 when n = 0: it is the start value again); interior values beyond the
// first (n > 2) take wm as well.  Scaled by s.
__device__ __forceinline__ float3 walk3(int k0, float f0, int k1, float f1, float s) {
  const int n = k1 > k0 ? k1 - k0 : k0 - k1;
  if (n == 0) return make_float3((f1 - f0) * s, 0.f, 0.f);
  const float wi = k1 > k0 ? s : -s;
  return k1 > k0 ? make_float3((1.f - f0) * s, n >= 2 ? wi : 0.f, f1 * s)
                 : make_float3(-f0 * s, n >= 2 ? wi : 0.f, (f1 - 1.f) * s);
}

// k0 and k1 of a walk packed in one word (indices below 32768)
__device__ __forceinline__ int pack_k(int k0, int k1) { return k0 | (k1 << 16); }

// Predicated 16-byte load through the read-only path into v, which keeps its
// value when p is false (no memory access then).  One instruction, so the
// loads of a walk issue back to back instead of behind branches; the kept
// value is finite image or sinogram data, and every caller gives it weight 0.
__device__ __forceinline__ void ldg4_keep(bool p, const float4* a, float4& v) {
  asm("{\n\t.reg .pred q;\n\t"
      "setp.ne.b32 q, %4, 0;\n\t"
      "@q ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%5];\n\t}"
      : "+f"(v.x), "+f"(v.y), "+f"(v.z), "+f"(v.w)
      : "r"((int)p), "l"(a));
}

// One walk for NZ z-tiles (float4 runs zoff[z] float4 past base): adds w0 cur
// + wm v[k0 + st] + we v[k1] (+ wm v for the further interior values) to acc
// and leaves v[k1] in cur.  v[k1] is loaded only when the walk moves (n >= 1;
// else it is cur), the first interior value only when there is one (n >= 2,
// into vm, which otherwise keeps an earlier value under weight 0): about two
// loads per footprint, and no branch unless it spans more than two steps.
#ifndef DDFAN_WALK_LOADS_FIRST
#define DDFAN_WALK_LOADS_FIRST 0
#endif
template <int NZ>
__device__ __forceinline__ void walk_nz(float (&acc)[NZ][4], float4 (&cur)[NZ], float4 (&vm)[NZ],
                                        const float4* base, size_t stride, const int (&zoff)[NZ], int k0, int k1,
                                        int kmax, const float4& wt) {
  const int dn = k1 - k0, st = dn > 0 ? 1 : -1, n = dn > 0 ? dn : -dn;
  const int km = min(max(k0 + st, 0), kmax);
  const float4* pm = base + (size_t)km * stride;
  const float4* pe = base + (size_t)k1 * stride;
#if DDFAN_WALK_LOADS_FIRST
  float4 ce[NZ];
#pragma unroll
  for (int z = 0; z < NZ; ++z) ce[z] = cur[z];
#pragma unroll
  for (int z = 0; z < NZ; ++z) ldg4_keep(n >= 2, pm + zoff[z], vm[z]);
#pragma unroll
  for (int z = 0; z < NZ; ++z) ldg4_keep(n >= 1, pe + zoff[z], ce[z]);
#pragma unroll
  for (int z = 0; z < NZ; ++z) {
    fma4(acc[z], wt.x, cur[z]);
    fma4(acc[z], wt.y, vm[z]);
    fma4(acc[z], wt.z, ce[z]);
    cur[z] = ce[z];
  }
#else
#pragma unroll
  for (int z = 0; z < NZ; ++z) ldg4_keep(n >= 2, pm + zoff[z], vm[z]);
#pragma unroll
  for (int z = 0; z < NZ; ++z) fma4(acc[z], wt.x, cur[z]);
#pragma unroll
  for (int z = 0; z < NZ; ++z) ldg4_keep(n >= 1, pe + zoff[z], cur[z]);
#pragma unroll
  for (int z = 0; z < NZ; ++z) {
    fma4(acc[z], wt.y, vm[z]);
    fma4(acc[z], wt.z, cur[z]);
  }
#endif
  for (int i = 2; i < n; ++i) {
    const float4* pi = base + (size_t)(k0 + i * st) * stride;
#pragma unroll
    for (int z = 0; z < NZ; ++z) fma4(acc[z], wt.y, __ldg(pi + zoff[z]));
  }
}

// ============================================================ forward projector

struct DdFwdArgs {
  const float4* img;   // masked image [YN][XN][P4]
  int P4;
  const ViewGeom* vg;
  const double2* fc;   // [PN][U+1] boundary lines
  const float* cvd;    // [PN][U] 1 / |dir.axis|
  const int* order;    // CTA row -> view, x-major first (null = identity)
  float* out;          // [slot][orow][ostride]
  int orow, ostride;
  int PN, U, Z, XN, YN;
  float dx;
  int zlo, zhi, zt0, nzt, row0;
  int nzc;             // most z-tiles per thread (launch shape; the kernel reads NZ)
  // fused OS-SART residual (AAPM_script/OSSART_AAPM.m:86-88); y null = plain projection
  const float* y;      // measured [views][U][ystride]
  const int* yview;    // slot -> measured view
  const float* rowsum; // [slot][U]
  const float* wgt;    // [slot][U] weight of the exact adjoint, or null
  int ystride;
};

// Lines of a forward chunk unrolled together, geometry elements (line,
// channel) a warp prepares per chunk, and z-tiles per thread.
#ifndef DDFAN_DD_FWD_UNROLL
#define DDFAN_DD_FWD_UNROLL 1
#endif
#ifndef DDFAN_DD_FWD_GEOM
#define DDFAN_DD_FWD_GEOM 256
#endif
// Ray sums: 0 = one running FP32 sum per ray; 1 = a sum per chunk of
// lines in registers, added to the totals, also in registers; 2 = chunk sums
// in registers, totals in dynamic shared memory (one slot per thread and
// value, so a chunk's sum is added with one load and one store per value).
// Chunk sums keep a 512-line ray's rounding at the level of ~CC terms; in
// registers they spill two channels per thread, in shared memory they cost
// the registers nothing.
#ifndef DDFAN_DD_FWD_PART
#define DDFAN_DD_FWD_PART 2
#endif
// geometry chunks per ray-sum chunk (DDFAN_DD_FWD_PART == 2)
#ifndef DDFAN_DD_FWD_FLUSH
#define DDFAN_DD_FWD_FLUSH 1
#endif
// most z-tiles per thread (1, 2 or 4; fewer when a call has fewer)
#ifndef DDFAN_DD_NZ
#define DDFAN_DD_NZ 4
#endif

// channels per thread of the direct forward projector for a z-lane count:
// two share the boundary value between them and the per-line decode
// (c3 subset: 2.16 -> 1.90 ms with one running sum per ray; with chunk sums
// the extra registers spill and the gain is gone)
#ifndef DDFAN_DD_FWD_CG
#define DDFAN_DD_FWD_CG 2
#endif
template <int ZL> struct DdFwdCG { static constexpr int v = ZL >= 4 ? DDFAN_DD_FWD_CG : (ZL == 2 ? 2 : 1); };

// z-tiles per thread of the direct kernels: each decoded footprint serves
// 4 slices per z-tile, so more z-tiles per thread means fewer instructions
// per slice (the measured lever: 1 -> 4 took a 96-view c3 subset's forward
// from 3.5 to 2.6 ms); at most the call's z-tiles
// (at most cap, the plan's tuned value)
inline int dd_nz(int nzt, int cap) { return nzt >= 4 && cap >= 4 ? 4 : (nzt >= 2 && cap >= 2 ? 2 : 1); }

template <int ZL, int CG, int NZ>
struct DdFwdTile {
  static constexpr int NT = 256, NW = NT / 32;
  static constexpr int GW = 32 / ZL;                  // channel groups per warp
  static constexpr int CWW = GW * CG;                 // channels per warp
  static constexpr int CW = NW * CWW;                 // channels per CTA
  static constexpr int CC = DDFAN_DD_FWD_GEOM / CWW;  // lines per geometry chunk
  static constexpr int UNROLL = DDFAN_DD_FWD_UNROLL;
  // dynamic shared memory of the ray totals (DDFAN_DD_FWD_PART == 2)
  static constexpr int DYN = DDFAN_DD_FWD_PART == 2 ? CG * NZ * 4 * NT * (int)sizeof(float) : 0;
};

// CTA = one view x CW channels x NZ z-tiles of 4*ZL slices; a thread owns CG
// consecutive channels x 4 slices in each of its NZ z-tiles and walks their
// footprints along each line, carrying the value at the boundary two channels
// share.  Every warp prepares the geometry of its own CWW channels (per chunk
// of CC lines: each channel's two cell indices and walk weights over
// 1 / footprint length, MultiSlicesProjGPU.cu:166-170) and synchronises with
// itself only, so warps interleave FP64 geometry with other warps' gathers.
template <int ZL, int CG, int NZ>
__device__ __forceinline__ void fwd_dd_body(const DdFwdArgs& a, int row, int cblk, int zgrp) {
  using T = DdFwdTile<ZL, CG, NZ>;
  constexpr int NW = T::NW, CWW = T::CWW, CW = T::CW, CC = T::CC;
  __shared__ double2 s_fc[NW][CWW + 1];
  __shared__ float4 s_w[NW][CC][CWW];  // (w0, wm, we) / length; k0 | k1 << 16 as int bits
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int zl = lane % ZL, gw = lane / ZL;
  if (row >= a.PN) return;  // uniform per CTA
  const int slot = a.order ? a.order[row] : row;
  const int p = slot;
  const int wc0 = cblk * CW + w * CWW;  // the warp's first channel
  if (wc0 >= a.U) return;  // uniform per warp; no CTA-wide barrier follows
  // z-tiles zt0 + zgrp * NZ + z of the call's nzt; block zb = zt * ZL + zl
  const int zt_first = a.zt0 + zgrp * NZ;
  int zbk[NZ], zoff[NZ];
  bool zok[NZ];
#pragma unroll
  for (int z = 0; z < NZ; ++z) {
    zbk[z] = (zt_first + z) * ZL + zl;
    zok[z] = zgrp * NZ + z < a.nzt && zbk[z] < a.P4;
    zoff[z] = zok[z] ? z * ZL : 0;  // a tile past the image reads the first one again (dropped)
  }
  const bool xm = a.vg[p].xmajor != 0;
  const int nl = xm ? a.XN : a.YN, N = xm ? a.YN : a.XN;
  for (int b = lane; b <= CWW; b += 32) s_fc[w][b] = a.fc[(size_t)p * (a.U + 1) + min(wc0 + b, a.U)];
  const bool active = (wc0 + gw * CG < a.U) && zok[0];
  // x-major views integrate along x columns (line = x, k = y), the others along y rows
  const size_t P4 = (size_t)a.P4;
  const size_t kstride = (xm ? (size_t)a.XN : 1) * P4;
  const size_t lstride = (xm ? 1 : (size_t)a.XN) * P4;
  const float4* img = a.img + (active ? zbk[0] : 0);
  float acc[CG][NZ][4];
  float4 vm[NZ];  // first interior values (kept between walks; see walk_nz)
#pragma unroll
  for (int z = 0; z < NZ; ++z) vm[z] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int j = 0; j < CG; ++j)
#pragma unroll
    for (int z = 0; z < NZ; ++z) acc[j][z][0] = acc[j][z][1] = acc[j][z][2] = acc[j][z][3] = 0.f;
  const double Nd = (double)N;
  const float dx = a.dx;
#if DDFAN_DD_FWD_PART == 2
  extern __shared__ float s_tot[];  // [CG * NZ * 4][NT]: this thread's totals at tid
  float* tot = s_tot + tid;
#pragma unroll
  for (int e = 0; e < CG * NZ * 4; ++e) tot[e * T::NT] = 0.f;
#endif
  __syncwarp();
  for (int ii0 = 0; ii0 < nl; ii0 += CC) {
    for (int e = lane; e < CC * CWW; e += 32) {
      const int col = e / CWW, j = e - col * CWW;
      const double di = (double)(ii0 + col);
      const double2 fa = s_fc[w][j], fb = s_fc[w][j + 1];
      const double c0 = fma(di, fa.x, fa.y), c1 = fma(di, fb.x, fb.y);
      const double cc0 = fmin(fmax(c0, 0.0), Nd), cc1 = fmin(fmax(c1, 0.0), Nd);
      const int k0 = min((int)cc0, N - 1), k1 = min((int)cc1, N - 1);
      const float f0 = (float)(cc0 - (double)k0), f1 = (float)(cc1 - (double)k1);
      const float inv = wc0 + j < a.U ? __frcp_rn((float)(c1 - c0) * dx) : 0.f;
      const float3 wt = walk3(k0, f0, k1, f1, inv);
      s_w[w][col][j] = make_float4(wt.x, wt.y, wt.z, __int_as_float(pack_k(k0, k1)));
    }
    __syncwarp();
    if (active) {
      const int ncol = min(CC, nl - ii0);
#if DDFAN_DD_FWD_PART == 1
      float part[CG][NZ][4];
#pragma unroll
      for (int j = 0; j < CG; ++j)
#pragma unroll
        for (int z = 0; z < NZ; ++z) part[j][z][0] = part[j][z][1] = part[j][z][2] = part[j][z][3] = 0.f;
#else
      float (&part)[CG][NZ][4] = acc;
#endif
#pragma unroll(T::UNROLL)
      for (int col = 0; col < ncol; ++col) {
        const float4* line = img + (size_t)(ii0 + col) * lstride;
        float4 cur[NZ];
        {
          const float4* p0 = line + (size_t)(__float_as_int(s_w[w][col][gw * CG].w) & 0xffff) * kstride;
#pragma unroll
          for (int z = 0; z < NZ; ++z) cur[z] = __ldg(p0 + zoff[z]);
        }
#pragma unroll
        for (int j = 0; j < CG; ++j) {
          const float4 wt = s_w[w][col][gw * CG + j];
          const int pk = __float_as_int(wt.w);
          walk_nz<NZ>(part[j], cur, vm, line, kstride, zoff, pk & 0xffff, pk >> 16, N - 1, wt);
        }
      }
#if DDFAN_DD_FWD_PART == 1
#pragma unroll
      for (int j = 0; j < CG; ++j)
#pragma unroll
        for (int z = 0; z < NZ; ++z)
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[j][z][s] += part[j][z][s];
#elif DDFAN_DD_FWD_PART == 2
      if ((ii0 / CC) % DDFAN_DD_FWD_FLUSH == DDFAN_DD_FWD_FLUSH - 1 || ii0 + CC >= nl) {
#pragma unroll
        for (int j = 0; j < CG; ++j)
#pragma unroll
          for (int z = 0; z < NZ; ++z)
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              float* t = tot + ((j * NZ + z) * 4 + s) * T::NT;
              *t += acc[j][z][s];
              acc[j][z][s] = 0.f;
            }
      }
#endif
    }
    __syncwarp();
  }
  if (!active) return;
#if DDFAN_DD_FWD_PART == 2
#pragma unroll
  for (int j = 0; j < CG; ++j)
#pragma unroll
    for (int z = 0; z < NZ; ++z)
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[j][z][s] = tot[((j * NZ + z) * 4 + s) * T::NT];
#endif
#pragma unroll
  for (int j = 0; j < CG; ++j) {
    const int u = wc0 + gw * CG + j;
    if (u >= a.U) break;
    const size_t e = (size_t)slot * a.U + u;
    const float cv = __ldg(a.cvd + e) * dx;
    float* o = a.out + ((size_t)slot * a.orow + u) * a.ostride;
    float rs = 0.f, wt = 1.f;
    const float* yv = nullptr;
    if (a.y) {
      rs = __ldg(a.rowsum + e);
      if (a.wgt) wt = __ldg(a.wgt + e);
      yv = a.y + ((size_t)__ldg(a.yview + slot) * a.U + u) * a.ystride;
    }
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
      if (!zok[z]) continue;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int zs = zbk[z] * 4 + s;
        if (zs < a.zlo || zs >= a.zhi) continue;
        float val = acc[j][z][s] * cv;
        if (yv) {
          // (y - A x) / rowSum where rowSum != 0, else A x (AAPM_script/OSSART_AAPM.m:88)
          val = rs != 0.f ? __fdiv_rn(__fsub_rn(__ldg(yv + zs), val), rs) : val;
          val *= wt;
        }
        o[zs] = val;
      }
    }
  }
}

// Grid order of the forward: with DDFAN_DD_FWD_ROWS_X the view rows run
// along grid x (dispatched first), so the CTAs in flight are every view of a
// few channel blocks -- rays at one distance from the centre, which miss the
// disk inside it -- instead of every channel block of a few views.  On a c3
// subset this cut the DRAM reads of the image from 2.05 to 1.33 GB per launch
// (L2 hits 74 -> 82 %) and the launch from 2.36 to 2.15 ms.
#ifndef DDFAN_DD_FWD_ROWS_X
#define DDFAN_DD_FWD_ROWS_X 1
#endif

// Allows a forward kernel its dynamic shared memory on the current device
// (above the 48 KB default with the static arrays).  Host-side, once per
// device, before any launch or capture.
template <typename K>
inline cudaError_t dd_allow_dyn(K kernel, int bytes) {
  return bytes > 0 ? cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) : cudaSuccess;
}

// One CTA per (view row, channel block, z-tile group) of one call.
template <int ZL, int CG, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_FWD_MIN_CTAS>::v)) k_fwd_dd(const __grid_constant__ DdFwdArgs a) {
#if DDFAN_DD_FWD_ROWS_X
  fwd_dd_body<ZL, CG, NZ>(a, a.row0 + (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z);
#else
  fwd_dd_body<ZL, CG, NZ>(a, a.row0 + (int)blockIdx.y, (int)blockIdx.x, (int)blockIdx.z);
#endif
}

// One launch over a work list of many calls (batched reconstructions): CTA
// b takes item {call, view row, channel block, z-tile group} = items[b].
template <int ZL, int CG, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_FWD_MIN_CTAS>::v)) k_fwd_dd_batch(const DdFwdArgs* __restrict__ args,
                                                                              const int4* __restrict__ items) {
  const int4 it = items[blockIdx.x];
#if DDFAN_DD_BATCH_ARGS_COPY
  const DdFwdArgs a = args[it.x];  // a local copy: its fields stay in registers
#else
  const DdFwdArgs& a = args[it.x];  // read in place (read-only, cached)
#endif
  fwd_dd_body<ZL, CG, NZ>(a, it.y, it.z, it.w);
}

// ============================================================ exact adjoint

struct DdAdjArgs {
  const float4* w;      // weighted residual [slot][U+1][P4], r_u / |dir_u.axis|, channel U = 0
  int P4;
  const ViewGeom* vg;
  const double2* fc;
  const float* tb;
  const uint16_t* lut;
  const int* order;
  const int* counts;
  float t0, invdt, dirt;
  int M;
  int PN, U, Z, XN, YN;
  double ocx, ocy, dx;
  BackEpi epi;
  int zt0, nzt;
  int nzc;  // most z-tiles per thread (launch shape; the kernel reads NZ)
};

// pixels per thread of the direct exact adjoint
#ifndef DDFAN_DD_BACK_VG
#define DDFAN_DD_BACK_VG 2
#endif

// Voxel tile of the direct exact adjoint: NG = 256/ZL groups as LT lines x
// SPL segments of VG consecutive voxels along the line.
template <int ZL>
struct DdBackTile {
  static constexpr int NT = 256;
  static constexpr int NG = NT / ZL;
  static constexpr int VG = DDFAN_DD_BACK_VG;
  static constexpr int SPL = 8;
  static constexpr int KT = SPL * VG;
  static constexpr int LT = NG / SPL;
};

// Transpose of k_fwd_dd, on the geometry of k_back_adj: pixel k of line ii
// receives sum_u w_u (fraction of footprint u inside [k, k+1]) = Q(beta(k+1))
// - Q(beta(k)), Q the channel prefix sum of w, beta the fractional boundary
// index of a pixel edge (bracket from the fan-tangent table, fraction from the
// FP64 boundary lines).  Here the difference is walked over w itself; a
// thread owns VG consecutive pixels of a line in NZ z-tiles, whose walks
// chain (the end of one is the start of the next).  Every warp brackets the
// edges of its own groups, ZL views at a time, and synchronises with itself
// only.
template <int ZL, bool XM, int NZ>
__device__ __forceinline__ void back_dd_body(const DdAdjArgs& a, int tile, int zgrp) {
  using T = DdBackTile<ZL>;
  constexpr int NT = T::NT, VG = T::VG, SPL = T::SPL, KT = T::KT, LT = T::LT;
  constexpr int NW = NT / 32, GW = 32 / ZL;  // warps, voxel groups per warp
  constexpr int VCW = ZL;                    // views per warp chunk (VCW * GW = 32)
  constexpr int NEG = VG + 1;                // edges per group
  constexpr int TBMAX = 1024, LUTMAX = 4096;
  __shared__ int2 s_geo[NW][VCW][GW][NEG];
  // per (view, pixel): the walk's weights and both edge cells packed, decoded
  // once for the ZL z-lanes that walk it
  __shared__ float4 s_wk[NW][VCW][GW][VG];
  __shared__ int s_p[NW][VCW];
  __shared__ float s_sgn[NW][VCW];
  __shared__ float s_tb[TBMAX];
  __shared__ uint16_t s_lut[LUTMAX];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int zl = lane % ZL, gw = lane / ZL;
  const int zt_first = a.zt0 + zgrp * NZ;
  int zbk[NZ], zoff[NZ];
  bool zok[NZ];
#pragma unroll
  for (int z = 0; z < NZ; ++z) {
    zbk[z] = (zt_first + z) * ZL + zl;
    zok[z] = zgrp * NZ + z < a.nzt && zbk[z] < a.P4;
    zoff[z] = zok[z] ? z * ZL : 0;  // a tile past the image reads the first one again (dropped)
  }
  const int nl = XM ? a.XN : a.YN, N = XM ? a.YN : a.XN;
  const int ntk = (N + KT - 1) / KT;
  const int tl = tile / ntk, tk = tile - tl * ntk;
  const int l0 = tl * LT, k0 = tk * KT;
  const int g = w * GW + gw;  // the thread's voxel group in the tile
  const int l = g / SPL, sg = g - l * SPL;
  const int ii = l0 + l, ks = k0 + sg * VG;
  const bool active = zok[0] && ii < nl && ks < N;
  for (int i = tid; i <= a.U; i += NT) s_tb[i] = a.tb[i];
  for (int i = tid; i < a.M; i += NT) s_lut[i] = a.lut[i];
  const int nx = a.counts[0];
  const int vbeg = XM ? 0 : nx, vend = XM ? nx : a.PN;
  float acc[VG][NZ][4];
  float4 vm[NZ];  // first interior values (kept between walks; see walk_nz)
#pragma unroll
  for (int z = 0; z < NZ; ++z) vm[z] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int v = 0; v < VG; ++v)
#pragma unroll
    for (int z = 0; z < NZ; ++z) acc[v][z][0] = acc[v][z][1] = acc[v][z][2] = acc[v][z][3] = 0.f;
  const size_t P4 = (size_t)a.P4;
  const size_t vstride = (size_t)(a.U + 1) * P4;
  const double ocl = XM ? a.ocx : a.ocy, ock = XM ? a.ocy : a.ocx;
  __syncthreads();  // the bracket tables; the rest of the kernel synchronises per warp
  const float tfirst = s_tb[0], tlast = s_tb[a.U];
  for (int v0 = vbeg; v0 < vend; v0 += VCW) {
    const int nvc = min(VCW, vend - v0);
    if (lane < nvc) {
      const int p = a.order[v0 + lane];
      s_p[w][lane] = p;
      s_sgn[w][lane] = a.vg[p].sgn;
    }
    __syncwarp();
    for (int e = lane; e < VCW * GW * NEG; e += 32) {
      const int vv = e / (GW * NEG), r = e - vv * (GW * NEG);
      const int gl = r / NEG, ke = r - gl * NEG;
      const int gg = w * GW + gl;
      const int li = l0 + gg / SPL, ck = k0 + (gg % SPL) * VG + ke;
      int b = 0;
      float frac = 0.f;
      if (vv < nvc && li < nl && ck <= N) {
        const int p = s_p[w][vv];
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
      s_geo[w][vv][gl][ke] = make_int2(b, __float_as_int(frac));
    }
    __syncwarp();
    // the walk of pixel v runs from edge v to edge v + 1 (chained: its end is
    // the next pixel's start)
    for (int e = lane; e < VCW * GW * VG; e += 32) {
      const int vv = e / (GW * VG), r = e - vv * (GW * VG);
      const int gl = r / VG, v = r - gl * VG;
      const int2 g0 = s_geo[w][vv][gl][v], g1 = s_geo[w][vv][gl][v + 1];
      const float3 ww = walk3(g0.x, __int_as_float(g0.y), g1.x, __int_as_float(g1.y), s_sgn[w][vv]);
      s_wk[w][vv][gl][v] = make_float4(ww.x, ww.y, ww.z, __int_as_float(pack_k(g0.x, g1.x)));
    }
    __syncwarp();
    if (active) {
      for (int vv = 0; vv < nvc; ++vv) {
        const float4* base = a.w + (size_t)s_p[w][vv] * vstride + zbk[0];
        const float4* wk = &s_wk[w][vv][gw][0];
        float4 cur[NZ];
        {
          const float4* p0 = base + (size_t)(__float_as_int(wk[0].w) & 0xffff) * P4;
#pragma unroll
          for (int z = 0; z < NZ; ++z) cur[z] = __ldg(p0 + zoff[z]);
        }
#pragma unroll
        for (int v = 0; v < VG; ++v) {
          const float4 g = wk[v];
          const int pk = __float_as_int(g.w);
          walk_nz<NZ>(acc[v], cur, vm, base, P4, zoff, pk & 0xffff, pk >> 16, a.U, g);
        }
      }
    }
    __syncwarp();
  }
  if (!active) return;
#pragma unroll
  for (int v = 0; v < VG; ++v) {
    const int kk = ks + v;
    if (kk >= N) break;
#pragma unroll
    for (int z = 0; z < NZ; ++z)
      if (zok[z]) back_store(a.epi, XM ? ii : kk, XM ? kk : ii, zbk[z], a.XN, a.Z, true, acc[v][z]);
  }
}

// One CTA per (voxel tile, z-tile group) of one call.
template <int ZL, bool XM, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_BACK_MIN_CTAS>::v)) k_back_dd(const __grid_constant__ DdAdjArgs a) {
  back_dd_body<ZL, XM, NZ>(a, (int)blockIdx.x, (int)blockIdx.z);
}

// The work-list launch: CTA b takes item {call, voxel tile, z-tile group} = items[b].
template <int ZL, bool XM, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_BACK_MIN_CTAS>::v)) k_back_dd_batch(const DdAdjArgs* __restrict__ args,
                                                                                const int4* __restrict__ items) {
  const int4 it = items[blockIdx.x];
#if DDFAN_DD_BATCH_ARGS_COPY
  const DdAdjArgs a = args[it.x];  // a local copy: its fields stay in registers
#else
  const DdAdjArgs& a = args[it.x];  // read in place (read-only, cached)
#endif
  back_dd_body<ZL, XM, NZ>(a, it.y, it.z);
}

// ============================================================ reference backprojector

struct DdRefArgs {
  const float4* q;     // residual [slot][U+1][P4] (unweighted), channel U = 0
  int P4;
  const ViewGeom* vg;
  int PN, U, Z, XN, YN;
  double ocx, ocy, dx, inv_sid, inv_dbeta, cnt;  // cnt = detCntIdx + 1 - 0.5
  BackEpi epi;
  int zt0, nzt;
  int nzc;  // most z-tiles per thread (launch shape; the kernel reads NZ)
};

// The reference backprojector's formula (AAPM_script/MultiSlicesBackGPU.cu:
// 115-184): angular detector coordinate alpha = asin(cross / (|s| l)),
// footprint half-width dx ddv / (2 l^2), weight dx l / ddv, coordinate
// alpha / dbeta + detCntIdx + 1, evaluated in FP64 once per (voxel, view) of
// a warp's voxels; the difference of the two channel prefix-sum samples is
// walked over the residual itself.  Voxel tile as the exact adjoint's (lines
// are image rows, k = x), VG voxels x NZ z-tiles per thread, ZL views per
// warp chunk, per-warp synchronisation only.
template <int ZL, int NZ>
__device__ __forceinline__ void ref_dd_body(const DdRefArgs& a, int tile, int zgrp) {
  using T = DdBackTile<ZL>;
  constexpr int NT = T::NT, VG = T::VG, SPL = T::SPL, KT = T::KT, LT = T::LT;
  constexpr int NW = NT / 32, GW = 32 / ZL;
  constexpr int VCW = ZL;  // views per warp chunk
  // per (view, voxel): the walk's weights (w0, wm, we) and both channel cells
  // packed (k0 | k1 << 16), decoded once here for the ZL z-lanes that walk it
  __shared__ float4 s_g[NW][VCW][GW][VG];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int zl = lane % ZL, gw = lane / ZL;
  const int zt_first = a.zt0 + zgrp * NZ;
  int zbk[NZ], zoff[NZ];
  bool zok[NZ];
#pragma unroll
  for (int z = 0; z < NZ; ++z) {
    zbk[z] = (zt_first + z) * ZL + zl;
    zok[z] = zgrp * NZ + z < a.nzt && zbk[z] < a.P4;
    zoff[z] = zok[z] ? z * ZL : 0;  // a tile past the image reads the first one again (dropped)
  }
  const int ntx = (a.XN + KT - 1) / KT;
  const int ty = tile / ntx, tx = tile - ty * ntx;
  const int y0 = ty * LT, x0 = tx * KT;
  const int g = w * GW + gw;
  const int l = g / SPL, sg = g - l * SPL;
  const int iy = y0 + l, ixs = x0 + sg * VG;
  const bool active = zok[0] && iy < a.YN && ixs < a.XN;
  float acc[VG][NZ][4];
  float4 vm[NZ];  // first interior values (kept between walks; see walk_nz)
#pragma unroll
  for (int z = 0; z < NZ; ++z) vm[z] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int v = 0; v < VG; ++v)
#pragma unroll
    for (int z = 0; z < NZ; ++z) acc[v][z][0] = acc[v][z][1] = acc[v][z][2] = acc[v][z][3] = 0.f;
  const double Ud = (double)a.U;
  const size_t P4 = (size_t)a.P4;
  const size_t vstride = (size_t)(a.U + 1) * P4;
  for (int v0 = 0; v0 < a.PN; v0 += VCW) {
    const int nvc = min(VCW, a.PN - v0);
    for (int e = lane; e < VCW * GW * VG; e += 32) {
      const int vv = e / (GW * VG), r = e - vv * (GW * VG);
      const int gl = r / VG, v = r - gl * VG;
      const int gg = w * GW + gl;
      const int yy = y0 + gg / SPL, xx = x0 + (gg % SPL) * VG + v;
      int2 ii = make_int2(0, 0);
      float2 ff = make_float2(0.f, 0.f);
      float wt = 0.f;
      if (vv < nvc && yy < a.YN && xx < a.XN && (!a.epi.mask || a.epi.mask[(size_t)yy * a.XN + xx] != 0)) {
        const ViewGeom& G = a.vg[v0 + vv];
        const double sx = G.sx, sy = G.sy;
        const double ddx = (xx - a.ocx) * a.dx - sx, ddy = (yy - a.ocy) * a.dx - sy;
        const double l2 = ddx * ddx + ddy * ddy;
        const double ln = sqrt(l2);
        const double alpha = asin((sy * ddx - sx * ddy) * a.inv_sid / ln);
        const double ddv = fabs(sx) > fabs(sy) ? ddx : ddy;
        const double da = ddv / l2 * a.dx * 0.5;
        wt = (float)(a.dx / ddv * ln);
        const double cL = fmin(fmax((alpha - da) * a.inv_dbeta + a.cnt, 0.0), Ud);
        const double cR = fmin(fmax((alpha + da) * a.inv_dbeta + a.cnt, 0.0), Ud);
        ii = make_int2(min((int)cL, a.U - 1), min((int)cR, a.U - 1));
        ff = make_float2((float)(cL - ii.x), (float)(cR - ii.y));
      }
      const float3 ww = walk3(ii.x, ff.x, ii.y, ff.y, wt);
      s_g[w][vv][gl][v] = make_float4(ww.x, ww.y, ww.z, __int_as_float(pack_k(ii.x, ii.y)));
    }
    __syncwarp();
    if (active) {
      for (int vv = 0; vv < nvc; ++vv) {
        const float4* base = a.q + (size_t)(v0 + vv) * vstride + zbk[0];
#pragma unroll
        for (int v = 0; v < VG; ++v) {
          const float4 g = s_g[w][vv][gw][v];
          const int pk = __float_as_int(g.w), k0 = pk & 0xffff, k1 = pk >> 16;
          float4 cur[NZ];
          const float4* p0 = base + (size_t)k0 * P4;
#pragma unroll
          for (int z = 0; z < NZ; ++z) cur[z] = __ldg(p0 + zoff[z]);
          walk_nz<NZ>(acc[v], cur, vm, base, P4, zoff, k0, k1, a.U, g);
        }
      }
    }
    __syncwarp();
  }
  if (!active) return;
#pragma unroll
  for (int v = 0; v < VG; ++v) {
    if (ixs + v >= a.XN) break;
#pragma unroll
    for (int z = 0; z < NZ; ++z)
      if (zok[z]) back_store(a.epi, ixs + v, iy, zbk[z], a.XN, a.Z, false, acc[v][z]);
  }
}

// One CTA per (voxel tile, z-tile group) of one call.
template <int ZL, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_BACK_MIN_CTAS>::v)) k_back_ref_dd(const __grid_constant__ DdRefArgs a) {
  ref_dd_body<ZL, NZ>(a, (int)blockIdx.x, (int)blockIdx.z);
}

// The work-list launch: CTA b takes item {call, voxel tile, z-tile group} = items[b].
template <int ZL, int NZ>
__global__ void __launch_bounds__(256, (DdMinCtas<NZ, DDFAN_DD_BACK_MIN_CTAS>::v)) k_back_ref_dd_batch(const DdRefArgs* __restrict__ args,
                                                                                    const int4* __restrict__ items) {
  const int4 it = items[blockIdx.x];
#if DDFAN_DD_BATCH_ARGS_COPY
  const DdRefArgs a = args[it.x];  // a local copy: its fields stay in registers
#else
  const DdRefArgs& a = args[it.x];  // read in place (read-only, cached)
#endif
  ref_dd_body<ZL, NZ>(a, it.y, it.z);
}

// ============================================================ staging

// dst[pix][z] = z < Z ? src[pix][z] * mask[pix] : 0 for z < Zp (mask null = 1):
// the masked image with its slices padded to a multiple of 4.
static __global__ void k_stage_image(const float* __restrict__ src, int Z, const uint8_t* __restrict__ mask,
                                     float* __restrict__ dst, int Zp, size_t npix) {
  const size_t n = npix * Zp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t pix = i / Zp;
    const int z = (int)(i - pix * Zp);
    float v = 0.f;
    if (z < Z) {
      v = src[pix * Z + z];
      if (mask && mask[pix] == 0) v = 0.f;
    }
    dst[i] = v;
  }
}

// dst[p][u][z] = src[p][u][z] * wgt[p][u] for u < U, z < Z; zero on the
// guard channel u = U and on padding slices (wgt null = 1).
static __global__ void k_stage_sino(const float* __restrict__ src, int Z, const float* __restrict__ wgt, int U,
                                    float* __restrict__ dst, int Zp, size_t PN) {
  const size_t n = PN * (U + 1) * Zp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / Zp;
    const int z = (int)(i - r * Zp);
    const size_t p = r / (U + 1);
    const int u = (int)(r - p * (U + 1));
    float v = 0.f;
    if (u < U && z < Z) {
      const size_t e = p * U + u;
      v = src[e * Z + z];
      if (wgt) v *= wgt[e];
    }
    dst[i] = v;
  }
}

// The published image of a solver that keeps masked voxels at 0 internally:
// out[pix][z] = mask ? x[pix][z] : x0[pix][z], clamped at 0 when the updates
// clamp (every update leaves a masked voxel at its initial value).
static __global__ void k_publish_masked(const float* __restrict__ x, int Zi, const float* __restrict__ x0,
                                        int Z, const uint8_t* __restrict__ mask, int clamp0,
                                        float* __restrict__ out, size_t npix) {
  const size_t n = npix * Z;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t pix = i / Z;
    const int z = (int)(i - pix * Z);
    float v;
    if (!mask || mask[pix] != 0) {
      v = x[pix * Zi + z];
    } else {
      v = x0[i];
      if (clamp0) v = fmaxf(v, 0.f);
    }
    out[i] = v;
  }
}

}  // namespace ddfan
