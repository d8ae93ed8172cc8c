// ddfan_rebin.cu -- helical-to-fan single-slice rebinning on the GPU.
//
// Same result, bit for bit, as the reference's CPU rebinning HelicalToFanImpl
// (AAPM_script/HelicalToFanFunc_mex.cpp:41-139, constants :160-164): for every
// target slice z and view ibeta of one rotation, raw helical view
// i = start + ibeta - 1 (start = floor((z - h/2) / deltaZ)) is interpolated
// linearly between detector rows at the row where the fan ray of channel j
// meets z, weighted by cos of the cone angle; a view any of whose channels
// falls outside the detector rows is zeroed whole.  Every floating-point
// operation of the reference is issued as one correctly rounded operation in
// the same order (no contraction into FMA), and the per-channel constants
// that the reference takes from the C library (cosf, atanf) are computed on
// the host with those same functions.
//
// Row validity without a reduction: within one output row (slice, view) the
// only channel-dependent input is SM_j = SO cos(angle_j) > 0, and every
// operation from SM_j to the interpolation row index is monotone, so the row
// is valid iff the channels with the smallest and the largest SM_j are.  The
// kernels evaluate those two once per row.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_plan.h"

namespace ddfan {
namespace {

struct RebinParams {
  const float* raw;    // raw views [view][W][H]; raw[0] is 1-based raw view view0
  long long view0;
  const float* sm;     // [W] SO * cosf((j - DetCenterW) * PerDetA), j 1-based
  const float* zpos;   // [SLN]
  const int* start;    // [SLN] floor((z - h/2) / deltaZ)
  float* out;
  float* views;
  const int* sstart;   // [nsorted] starts >= 0 in ascending order
  const int* sslice;   // [nsorted] their slices
  int nsorted, chunks; // chunks: warps per raw view (32 slices each) to cover its slices
  int SLN, T, W, H;    // T = DefTimes
  float SD, SD2, PH, DCH, deltaZ, delta, BV, twopi, sm_lo, sm_hi;
};

// fractional detector row of the ray with SM at height offset n (1-based, as the reference)
__device__ __forceinline__ float rebin_dv(const RebinParams& p, float n, float sm, float* v) {
  const float tanv = __fdiv_rn(n, sm);
  *v = __fmul_rn(p.SD, tanv);
  return __fadd_rn(__fdiv_rn(__fadd_rn(p.DCH, *v), p.PH), 1.0f);
}

__device__ __forceinline__ bool rebin_in_rows(const RebinParams& p, float dv) {
  return dv >= 1.0f && dv < (float)p.H;  // 1 <= floor(dv) <= H - 1
}

struct RebinRow {
  const float* col;  // raw view of this row, channel 0
  float n;           // z - zz, zz = (i - 1) deltaZ the height of raw view i
  bool ok;           // computed and every channel inside the detector rows
};

__device__ __forceinline__ RebinRow rebin_row(const RebinParams& p, int s, int ib) {
  RebinRow r;
  r.col = nullptr;
  r.n = 0.f;
  r.ok = false;
  const int st = p.start[s];
  const long long i = (long long)st + ib;  // 1-based raw view
  if (st < 0 || i < 1) return r;           // the reference's size_t loop skips these
  const float zz = __fmul_rn((float)(i - 1), p.deltaZ);
  r.n = __fsub_rn(p.zpos[s], zz);
  float v;
  r.ok = rebin_in_rows(p, rebin_dv(p, r.n, p.sm_lo, &v)) && rebin_in_rows(p, rebin_dv(p, r.n, p.sm_hi, &v));
  r.col = p.raw + (size_t)(i - p.view0) * p.W * p.H;
  return r;
}

__device__ __forceinline__ float rebin_view_angle(const RebinParams& p, int s, int ib) {
  const int st = p.start[s];
  const long long i = (long long)st + ib;
  if (st < 0 || i < 1) return 0.f;
  float lam = __fadd_rn(__fmul_rn((float)(i - 1), p.delta), p.BV);
  while (lam > p.twopi) lam = __fsub_rn(lam, p.twopi);
  return lam;
}

// one output sample of a valid row.  VEC: detector columns start 16-byte
// aligned (DetHeight % 4 == 0); the two rows then come from one 16-byte load
// (one L1 request per sample instead of two), plus a 4-byte load when they
// straddle two 16-byte words.
template <bool VEC>
__device__ __forceinline__ float rebin_sample(const RebinParams& p, const RebinRow& r, int j) {
  float v;
  const float dv = rebin_dv(p, r.n, __ldg(p.sm + j), &v);
  int idv = (int)floorf(dv);
  idv = min(max(idv, 1), p.H - 1);  // already so for a valid row; keeps the loads in bounds regardless
  const float t = __fsub_rn(dv, (float)idv);
  const float* colj = r.col + (size_t)j * p.H;
  float d0, d1;
  if (VEC) {
    // e + 3 <= H - 1 because idv - 1 <= H - 2 and H % 4 == 0
    const int e = (idv - 1) & ~3, q = (idv - 1) - e;
    const float4 w = __ldg(reinterpret_cast<const float4*>(colj + e));
    d0 = q == 0 ? w.x : q == 1 ? w.y : q == 2 ? w.z : w.w;
    d1 = q == 0 ? w.y : q == 1 ? w.z : q == 2 ? w.w : __ldg(colj + e + 4);
  } else {
    d0 = __ldg(colj + idv - 1);
    d1 = __ldg(colj + idv);
  }
  const float temp = __fadd_rn(__fmul_rn(d0, __fsub_rn(1.0f, t)), __fmul_rn(d1, t));
  const float cosv = __fdiv_rn(p.SD, __fsqrt_rn(__fadd_rn(p.SD2, __fmul_rn(v, v))));
  return __fmul_rn(cosv, temp);
}

// first index k in [0, n) with a[k] >= x (a ascending)
__device__ __forceinline__ int lower_bound_int(const int* a, int n, long long x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if ((long long)__ldg(a + m) < x) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// Mex layout out[s][ib][j], views[s][ib], traversed along raw views: warp
// (view, chunk) takes raw view i and up to 32 of the slices that read it --
// those with start in [i - T + 1, i], consecutive in start order -- one per
// lane, each making its row ib = i - start.  The 32 lanes read one detector
// column at neighbouring heights (a few sectors per load instead of one
// sector per lane), every lane has work, and the warps of neighbouring raw
// views run side by side and share those views in L2.  Each warp gathers a
// 32-slice x 32-channel tile in shared memory and stores it as 128-byte row
// pieces.  Rows no raw view >= 1 reaches are written by k_rebin_unvisited.
template <bool VEC>
__global__ void __launch_bounds__(256) k_rebin_diag(RebinParams p, long long vlo, long long vhi) {
  __shared__ float tile[8][32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long gw = (long long)blockIdx.x * 8 + warp;
  const long long i = vlo + gw / p.chunks;  // 1-based raw view, >= vlo >= 1
  const int q = (int)(gw % p.chunks);
  if (i > vhi) return;  // uniform per warp; no block-wide barrier follows
  const int a = lower_bound_int(p.sstart, p.nsorted, i - p.T + 1);
  const int b = lower_bound_int(p.sstart, p.nsorted, i + 1);
  const int k = a + 32 * q + lane;
  const bool act = k < b;
  const unsigned amask = __ballot_sync(0xffffffffu, act);
  if (!amask) return;
  const int s = act ? __ldg(p.sslice + k) : 0;
  const int ib = act ? (int)(i - __ldg(p.sstart + k)) : 0;
  float(*t)[33] = tile[warp];
  RebinRow r;
  r.n = act ? __fsub_rn(__ldg(p.zpos + s), __fmul_rn((float)(i - 1), p.deltaZ)) : 0.f;
  float vtmp;
  r.ok = act && rebin_in_rows(p, rebin_dv(p, r.n, p.sm_lo, &vtmp)) &&
         rebin_in_rows(p, rebin_dv(p, r.n, p.sm_hi, &vtmp));
  r.col = p.raw + (size_t)(i - p.view0) * p.W * p.H;
  if (act) {
    float lam = __fadd_rn(__fmul_rn((float)(i - 1), p.delta), p.BV);
    while (lam > p.twopi) lam = __fsub_rn(lam, p.twopi);
    p.views[(size_t)s * p.T + ib] = lam;
  }
  for (int j0 = 0; j0 < p.W; j0 += 32) {
    const int nc = min(32, p.W - j0);
#pragma unroll 4
    for (int c = 0; c < 32; ++c) t[lane][c] = (r.ok && c < nc) ? rebin_sample<VEC>(p, r, j0 + c) : 0.f;
    __syncwarp();
    for (unsigned m = amask; m; m &= m - 1) {
      const int qq = __ffs(m) - 1;
      const int sq = __shfl_sync(0xffffffffu, s, qq);
      const int ibq = __shfl_sync(0xffffffffu, ib, qq);
      if (lane < nc) p.out[((size_t)sq * p.T + ibq) * p.W + j0 + lane] = t[qq][lane];
    }
    __syncwarp();
  }
}

// Rows the reference never computes and leaves zero: every row of a slice
// with start < 0, row 0 of a slice with start == 0 (its raw view would be 0).
__global__ void __launch_bounds__(256) k_rebin_unvisited(RebinParams p) {
  const int s = blockIdx.x;
  const int st = p.start[s];
  const int nz = st < 0 ? p.T : (st == 0 ? 1 : 0);
  for (int ib = 0; ib < nz; ++ib) {
    float* o = p.out + ((size_t)s * p.T + ib) * p.W;
    for (int j = threadIdx.x; j < p.W; j += blockDim.x) o[j] = 0.f;
    if (threadIdx.x == 0) p.views[(size_t)s * p.T + ib] = 0.f;
  }
}

// Routine layout (after HelicalToFan_routine.m:44-45 permutes, the solver's
// sinogram layout): out[ib][j][s], views[ib][s].  A CTA owns 32 slices of one
// view; warps compute rows (lanes over 32 channels) into a shared tile, then
// store it transposed with lanes over slices (128-byte rows).
template <bool VEC>
__global__ void __launch_bounds__(256) k_rebin_routine(RebinParams p) {
  __shared__ float tile[32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ib = blockIdx.x;
  const int s0 = blockIdx.y * 32;
  RebinRow rows[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int s = s0 + warp * 4 + q;
    if (s < p.SLN) {
      rows[q] = rebin_row(p, s, ib);
    } else {
      rows[q].ok = false;
      rows[q].col = nullptr;
      rows[q].n = 0.f;
    }
  }
  if (warp == 0 && s0 + lane < p.SLN)
    p.views[(size_t)ib * p.SLN + s0 + lane] = rebin_view_angle(p, s0 + lane, ib);
  const int ns = min(32, p.SLN - s0);
  for (int j0 = 0; j0 < p.W; j0 += 32) {
    const int j = j0 + lane;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      tile[warp * 4 + q][lane] = (rows[q].ok && j < p.W) ? rebin_sample<VEC>(p, rows[q], j) : 0.f;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int jj = j0 + warp * 4 + q;
      if (jj < p.W && lane < ns) p.out[((size_t)ib * p.W + jj) * p.SLN + s0 + lane] = tile[lane][warp * 4 + q];
    }
    __syncthreads();
  }
}

// DICOM-CT-PD stored pixels -> raw views: out[v'][k] = (float)pix[v][k],
// v' = n - 1 - v when reversing (readProj.m:54 flips the view order), for the
// W x H pixels k of a view (DICOM rows = detector columns, columns = detector
// rows: already the [channel][row] layout).  8 pixels per thread and step.
__global__ void __launch_bounds__(256) k_ctpd_views(const uint16_t* __restrict__ pix, long long n, long long per,
                                                    int reverse, float* __restrict__ out) {
  const long long total = n * per;
  const long long stride = (long long)gridDim.x * blockDim.x * 8;
  const bool vec = (per % 8) == 0;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 8; i < total; i += stride) {
    const long long v = i / per, k = i - v * per;
    const long long o = (reverse ? (n - 1 - v) : v) * per + k;
    if (vec) {
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(pix + i));
      const uint32_t w[4] = {q.x, q.y, q.z, q.w};
      float4 a, b;
      a.x = (float)(w[0] & 0xffffu); a.y = (float)(w[0] >> 16);
      a.z = (float)(w[1] & 0xffffu); a.w = (float)(w[1] >> 16);
      b.x = (float)(w[2] & 0xffffu); b.y = (float)(w[2] >> 16);
      b.z = (float)(w[3] & 0xffffu); b.w = (float)(w[3] >> 16);
      reinterpret_cast<float4*>(out + o)[0] = a;
      reinterpret_cast<float4*>(out + o)[1] = b;
    } else {
      for (int j = 0; j < 8 && i + j < total; ++j) {
        const long long ij = i + j, vj = ij / per, kj = ij - vj * per;
        out[(reverse ? (n - 1 - vj) : vj) * per + kj] = (float)pix[ij];
      }
    }
  }
}

struct RebinHost {
  RebinParams p;
  std::vector<float> sm;
  std::vector<int> start;
  std::vector<int> sstart, sslice;  // slices with start >= 0, by ascending start
  long long lo = 0, hi = -1;  // 1-based raw views the computed rows read (empty when hi < lo)
};

// Host constants exactly as HelicalToFan (HelicalToFanFunc_mex.cpp:160-164) and
// HelicalToFanImpl (:66, :80-84) compute them, plus argument checks.
int rebin_prepare(RebinHost& h, long long nViews, const float* zPos, int SLN, float SD, float SO,
                  float BVAngle, int DetWidth, int DetHeight, float PerDetW, float PerDetH,
                  int DefTimes, float DetCenterW, float SpiralPitchFactor) {
  if (!zPos) return set_err(DDFAN_ERR_ARG, "HelicalToFan: null zPos");
  if (SLN < 1 || DetWidth < 1 || DetHeight < 2 || DefTimes < 1 || nViews < 1 || SLN > 65535)
    return set_err(DDFAN_ERR_ARG, "HelicalToFan: bad sizes (SLN=%d DetWidth=%d DetHeight=%d DefTimes=%d views=%lld)",
                   SLN, DetWidth, DetHeight, DefTimes, nViews);
  const float PerDetA = 2.0f * atanf(PerDetW / SD * 0.5f);
  const float delta = 2.0 * M_PI / DefTimes;
  const float DetCenterHreal = (DetHeight - 1.0) * 0.5 / PerDetH;
  const float hh = SpiralPitchFactor * PerDetH * DetHeight * SO / SD;
  const float deltaZ = hh / DefTimes;
  if (!std::isfinite(deltaZ) || !(std::fabs(deltaZ) > 0.f) || !std::isfinite(SD) || !std::isfinite(PerDetH) ||
      PerDetH == 0.f)
    return set_err(DDFAN_ERR_ARG, "HelicalToFan: degenerate geometry (deltaZ=%g SD=%g PerDetH=%g)", deltaZ, SD,
                   PerDetH);
  h.sm.resize(DetWidth);
  float lo = INFINITY, hi = -INFINITY;
  for (int j = 1; j <= DetWidth; ++j) {
    const float ang = (j - DetCenterW) * PerDetA;
    const float SM = SO * cosf(ang);
    h.sm[j - 1] = SM;
    lo = std::min(lo, SM);
    hi = std::max(hi, SM);
  }
  // the one-pair row test needs every SM_j finite and of one sign
  if (!std::isfinite(lo) || !std::isfinite(hi) || !((lo > 0.f) || (hi < 0.f)))
    return set_err(DDFAN_ERR_UNSUPPORTED, "HelicalToFan: channel fan angles reach 90 degrees (SO*cos in [%g, %g])",
                   lo, hi);
  h.start.resize(SLN);
  h.lo = (long long)1 << 62;
  h.hi = -1;
  for (int s = 0; s < SLN; ++s) {
    const float z = zPos[s];
    const float q = floorf((z - hh * 0.5f) / deltaZ);
    if (!std::isfinite(q) || std::fabs(q) > 1.0e9f)
      return set_err(DDFAN_ERR_ARG, "HelicalToFan: zPos[%d] = %g is far outside the scan", s, z);
    const int st = (int)q;
    h.start[s] = st;
    if (st < 0) continue;  // the reference leaves such a slice zero
    const long long last = (long long)st + DefTimes - 1;
    if (last > nViews)
      return set_err(DDFAN_ERR_ARG, "HelicalToFan: slice %d (z = %g) needs raw view %lld, only %lld given", s, z, last,
                     nViews);
    if (last >= 1) {
      h.lo = std::min(h.lo, std::max(1LL, (long long)st));
      h.hi = std::max(h.hi, last);
    }
  }
  if (h.hi < h.lo) h.lo = 1, h.hi = 0;
  // slices in start order, and how many of them one raw view serves at most
  std::vector<int> idx;
  for (int s = 0; s < SLN; ++s)
    if (h.start[s] >= 0) idx.push_back(s);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return h.start[a] < h.start[b]; });
  h.sslice = idx;
  h.sstart.resize(idx.size());
  for (size_t k = 0; k < idx.size(); ++k) h.sstart[k] = h.start[idx[k]];
  int most = 0;
  for (size_t k0 = 0, k1 = 0; k0 < idx.size(); ++k0) {
    while (k1 < idx.size() && (long long)h.sstart[k1] <= (long long)h.sstart[k0] + DefTimes - 1) ++k1;
    most = std::max(most, (int)(k1 - k0));
  }
  RebinParams& p = h.p;
  p = RebinParams{};
  p.nsorted = (int)idx.size();
  p.chunks = std::max(1, (most + 31) / 32);
  p.SLN = SLN; p.T = DefTimes; p.W = DetWidth; p.H = DetHeight;
  p.SD = SD; p.SD2 = SD * SD; p.PH = PerDetH; p.DCH = DetCenterHreal;
  p.deltaZ = deltaZ; p.delta = delta; p.BV = BVAngle; p.twopi = (float)(2 * M_PI);
  p.sm_lo = lo; p.sm_hi = hi;
  return DDFAN_OK;
}

// layout 0 (mex layouts): raw-view-order traversal, plus the rows it never
// visits; layout 1 (slices last): one CTA per (32 slices, view).
int rebin_launch(const RebinHost& h, int layout, cudaStream_t st) {
  const RebinParams& p = h.p;
  // 16-byte loads need 16-byte aligned columns: DetHeight % 4 == 0 and an aligned base
  const bool vec = p.H % 4 == 0 && (reinterpret_cast<uintptr_t>(p.raw) & 15) == 0;
  if (layout == 0) {
    k_rebin_unvisited<<<p.SLN, 256, 0, st>>>(p);
    if (h.hi >= h.lo && p.nsorted > 0) {
      const long long warps = (h.hi - h.lo + 1) * (long long)p.chunks;
      const long long ctas = (warps + 7) / 8;
      if (ctas > 0x7fffffffLL)
        return set_err(DDFAN_ERR_UNSUPPORTED, "HelicalToFan: %lld raw views in one call", h.hi - h.lo + 1);
      if (vec) k_rebin_diag<true><<<(unsigned)ctas, 256, 0, st>>>(p, h.lo, h.hi);
      else k_rebin_diag<false><<<(unsigned)ctas, 256, 0, st>>>(p, h.lo, h.hi);
    }
  } else {
    dim3 grid(p.T, (p.SLN + 31) / 32);
    if (vec) k_rebin_routine<true><<<grid, 256, 0, st>>>(p);
    else k_rebin_routine<false><<<grid, 256, 0, st>>>(p);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "HelicalToFan launch: %s", cudaGetErrorString(e));
  return DDFAN_OK;
}

// small host->device uploads of the per-channel and per-slice tables into one buffer
// Pinned staging for the small per-call tables, one per device: a pageable
// source would make cudaMemcpyAsync wait for the stream, leaving the GPU idle
// between back-to-back calls.  The buffer is reused once the previous call's
// copy out of it has completed (its event), so a call never waits for kernels.
struct Staging {
  std::mutex m;
  unsigned char* host = nullptr;
  size_t cap = 0;
  cudaEvent_t copied = nullptr;
};
constexpr int kMaxStagingDevices = 64;
Staging g_staging[kMaxStagingDevices];

int rebin_tables(RebinHost& h, const float* zPos, void** buf, cudaStream_t st) {
  const int W = h.p.W, SLN = h.p.SLN;
  const size_t b_sm = ((sizeof(float) * W + 255) / 256) * 256;
  const size_t b_z = ((sizeof(float) * SLN + 255) / 256) * 256;
  const size_t b_i = ((sizeof(int) * SLN + 255) / 256) * 256;
  const size_t bytes = b_sm + b_z + 3 * b_i;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxStagingDevices) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "HelicalToFan: no usable current device");
  }
  int rc = dev_alloc(buf, bytes, st);
  if (rc) return rc;
  unsigned char* b = static_cast<unsigned char*>(*buf);
  Staging& sg = g_staging[dev];
  std::lock_guard<std::mutex> lock(sg.m);
  cudaError_t e = cudaSuccess;
  if (!sg.copied) e = cudaEventCreateWithFlags(&sg.copied, cudaEventDisableTiming);
  else e = cudaEventSynchronize(sg.copied);  // the previous upload has left the buffer
  if (e == cudaSuccess && sg.cap < bytes) {
    if (sg.host) cudaFreeHost(sg.host);
    sg.host = nullptr;
    sg.cap = 0;
    e = cudaHostAlloc(reinterpret_cast<void**>(&sg.host), bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) sg.cap = bytes;
  }
  if (e == cudaSuccess) {
    std::memcpy(sg.host, h.sm.data(), sizeof(float) * W);
    std::memcpy(sg.host + b_sm, zPos, sizeof(float) * SLN);
    std::memcpy(sg.host + b_sm + b_z, h.start.data(), sizeof(int) * SLN);
    if (!h.sstart.empty()) {
      std::memcpy(sg.host + b_sm + b_z + b_i, h.sstart.data(), sizeof(int) * h.sstart.size());
      std::memcpy(sg.host + b_sm + b_z + 2 * b_i, h.sslice.data(), sizeof(int) * h.sslice.size());
    }
    e = cudaMemcpyAsync(b, sg.host, bytes, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaEventRecord(sg.copied, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    dev_free(*buf, st);
    *buf = nullptr;
    return set_err(DDFAN_ERR_CUDA, "HelicalToFan table upload: %s", cudaGetErrorString(e));
  }
  h.p.sm = reinterpret_cast<const float*>(b);
  h.p.zpos = reinterpret_cast<const float*>(b + b_sm);
  h.p.start = reinterpret_cast<const int*>(b + b_sm + b_z);
  h.p.sstart = reinterpret_cast<const int*>(b + b_sm + b_z + b_i);
  h.p.sslice = reinterpret_cast<const int*>(b + b_sm + b_z + 2 * b_i);
  return DDFAN_OK;
}

}  // namespace
}  // namespace ddfan

using namespace ddfan;

extern "C" DDFAN_API int ddfan_helical_to_fan_dev(const float* d_proj, long long nViews, const float* zPos, int SLN,
                                                  float SD, float SO, float BVAngle, int DetWidth, int DetHeight,
                                                  float PerDetW, float PerDetH, int DefTimes, float DetCenterW,
                                                  float SpiralPitchFactor, int layout, float* d_Proj,
                                                  float* d_Views, void* stream) {
  if (!d_proj || !d_Proj || !d_Views) return set_err(DDFAN_ERR_ARG, "helical_to_fan_dev: null argument");
  if (layout != 0 && layout != 1) return set_err(DDFAN_ERR_ARG, "helical_to_fan_dev: layout %d", layout);
  RebinHost h;
  int rc = rebin_prepare(h, nViews, zPos, SLN, SD, SO, BVAngle, DetWidth, DetHeight, PerDetW, PerDetH, DefTimes,
                         DetCenterW, SpiralPitchFactor);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  void* tables = nullptr;
  if ((rc = rebin_tables(h, zPos, &tables, st))) return rc;
  h.p.raw = d_proj;
  h.p.view0 = 1;
  h.p.out = d_Proj;
  h.p.views = d_Views;
  rc = rebin_launch(h, layout, st);
  dev_free(tables, st);
  return rc;
}

extern "C" DDFAN_API int ddfan_HelicalToFan(float* Proj, float* Views, const float* proj, long long nViews,
                                            const float* zPos, int SLN, float SD, float SO, float BVAngle,
                                            int DetWidth, int DetHeight, float PerDetW, float PerDetH,
                                            int DefTimes, float DetCenterW, float SpiralPitchFactor) {
  if (!Proj || !Views || !proj) return set_err(DDFAN_ERR_ARG, "HelicalToFan: null argument");
  RebinHost h;
  int rc = rebin_prepare(h, nViews, zPos, SLN, SD, SO, BVAngle, DetWidth, DetHeight, PerDetW, PerDetH, DefTimes,
                         DetCenterW, SpiralPitchFactor);
  if (rc) return rc;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "HelicalToFan: cudaStreamCreate failed");
  }
  const size_t view_elems = (size_t)DetWidth * DetHeight;
  const size_t nraw = h.hi >= h.lo ? (size_t)(h.hi - h.lo + 1) : 0;
  const size_t out_elems = (size_t)SLN * DefTimes * DetWidth;
  void *d_raw = nullptr, *d_out = nullptr, *d_views = nullptr, *tables = nullptr;
  rc = dev_alloc(&d_raw, std::max<size_t>(1, nraw) * view_elems * sizeof(float), st);
  if (!rc) rc = dev_alloc(&d_out, out_elems * sizeof(float), st);
  if (!rc) rc = dev_alloc(&d_views, (size_t)SLN * DefTimes * sizeof(float), st);
  if (!rc) rc = rebin_tables(h, zPos, &tables, st);
  if (!rc && nraw) {
    // only the raw views some computed row reads travel to the device
    cudaError_t e = cudaMemcpyAsync(d_raw, proj + (size_t)(h.lo - 1) * view_elems, nraw * view_elems * sizeof(float),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = set_err(DDFAN_ERR_CUDA, "HelicalToFan: raw upload: %s", cudaGetErrorString(e));
    }
  }
  if (!rc) {
    h.p.raw = static_cast<const float*>(d_raw);
    h.p.view0 = nraw ? h.lo : 1;
    h.p.out = static_cast<float*>(d_out);
    h.p.views = static_cast<float*>(d_views);
    rc = rebin_launch(h, 0, st);
  }
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(Proj, d_out, out_elems * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(Views, d_views, (size_t)SLN * DefTimes * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = set_err(DDFAN_ERR_CUDA, "HelicalToFan: %s", cudaGetErrorString(e));
    }
  }
  dev_free(tables, st);
  dev_free(d_views, st);
  dev_free(d_out, st);
  dev_free(d_raw, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return rc;
}

extern "C" DDFAN_API int ddfan_ctpd_views_to_raw(const uint16_t* d_pix, long long nViews, int W, int H, int reverse,
                                                 float* d_proj, void* stream) {
  if (!d_pix || !d_proj) return set_err(DDFAN_ERR_ARG, "ctpd_views_to_raw: null argument");
  if (nViews < 1 || W < 1 || H < 1) return set_err(DDFAN_ERR_ARG, "ctpd_views_to_raw: bad sizes");
  const long long per = (long long)W * H;
  if ((per % 8) == 0 &&
      ((reinterpret_cast<uintptr_t>(d_pix) & 15) != 0 || (reinterpret_cast<uintptr_t>(d_proj) & 15) != 0))
    return set_err(DDFAN_ERR_ARG, "ctpd_views_to_raw: buffers must be 16-byte aligned");
  const long long work = (nViews * per + 7) / 8;
  const int blocks = (int)std::min<long long>((work + 255) / 256, 148LL * 8);
  k_ctpd_views<<<std::max(blocks, 1), 256, 0, (cudaStream_t)stream>>>(d_pix, nViews, per, reverse ? 1 : 0, d_proj);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "ctpd_views_to_raw launch: %s", cudaGetErrorString(e));
  return DDFAN_OK;
}
