// ddfan_solver.cu -- mex-compatible host entry points and the device-resident
// OS-SART / FISTA solver of libddfan.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_kernels.cuh"
#include "ddfan_plan.h"
#include "ddfan_ps.h"
#include "ddfan_solver.h"

namespace ddfan {

namespace {

struct PlanPtr {
  Plan* p = nullptr;
  ~PlanPtr() { plan_free(p); }
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  cudaStream_t st = nullptr;  // allocation and release are ordered on this stream
  explicit DevBuf(cudaStream_t s = nullptr) : st(s) {}
  ~DevBuf() { dev_free(p, st); }
  int alloc(size_t n) { return dev_alloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T), st); }
};

#define DDFAN_CK(call)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return set_err(DDFAN_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                     __LINE__);                                                                \
  } while (0)

// Slabs of slices per device, as startIdx describes them
// (AAPM_script/DD2MutiSlices.m:95-101, MultiSlicesProjGPU.cu:500-514).
int slabs_of(const int32_t* startIdx, int n, int SLN, std::vector<std::pair<int, int>>& out) {
  out.clear();
  if (!startIdx || n <= 0) {
    out.emplace_back(0, SLN);
    return DDFAN_OK;
  }
  for (int k = 0; k < n; ++k) {
    const int a = startIdx[k], b = k + 1 < n ? startIdx[k + 1] : SLN;
    if (a < 0 || b > SLN || a > b) return set_err(DDFAN_ERR_ARG, "startIdx[%d]=%d: slabs must be increasing within [0, %d]", k, a, SLN);
    if (k == 0 && a != 0) return set_err(DDFAN_ERR_ARG, "startIdx[0] must be 0");
    if (b > a) out.emplace_back(a, b);
  }
  return DDFAN_OK;
}

// gather slices [a, b) of a [rows][SLN] array into [rows][b - a]
void gather_slab(const float* src, size_t rows, int SLN, int a, int b, std::vector<float>& dst) {
  const int n = b - a;
  dst.resize(rows * n);
  for (size_t r = 0; r < rows; ++r) std::memcpy(&dst[r * n], src + r * SLN + a, sizeof(float) * n);
}

void scatter_slab(const std::vector<float>& src, size_t rows, int SLN, int a, int b, float* dst) {
  const int n = b - a;
  for (size_t r = 0; r < rows; ++r) std::memcpy(dst + r * SLN + a, &src[r * n], sizeof(float) * n);
}

int device_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace

// One slab of a mex-style call on one device: upload, project or backproject
// (per distinct angle list, or slice-major), download.
static int mex_slab(bool forward, const PlanDesc& d, const float* angs, int PN, const float* in,
                    float* out, int back_mode) {
  PlanPtr P;
  int rc = plan_create(&P.p, d);
  if (rc) return rc;
  Plan& p = *P.p;
  DeviceGuard g(p.device);
  const size_t V = (size_t)p.XN * p.YN * p.Z, S = (size_t)PN * p.U * p.Z;
  DevBuf<float> din, dout;
  if ((rc = din.alloc(forward ? V : S)) || (rc = dout.alloc(forward ? S : V))) return rc;
  DDFAN_CK(cudaMemcpy(din.p, in, sizeof(float) * (forward ? V : S), cudaMemcpyHostToDevice));
  // per-slice angle lists: one launch group per distinct list, or the
  // slice-major kernels
  DevBuf<float> dang;
  if ((rc = dang.alloc((size_t)PN * p.Z))) return rc;
  DDFAN_CK(cudaMemcpy(dang.p, angs, sizeof(float) * PN * p.Z, cudaMemcpyHostToDevice));
  rc = forward ? proj_dev_per_slice(p, dang.p, angs, PN, din.p, dout.p, 0)
               : back_dev_per_slice(p, dang.p, angs, PN, din.p, dout.p, back_mode, 0);
  if (rc) return rc;
  DDFAN_CK(cudaDeviceSynchronize());
  DDFAN_CK(cudaMemcpy(out, dout.p, sizeof(float) * (forward ? S : V), cudaMemcpyDeviceToHost));
  return DDFAN_OK;
}

// Slabs [startIdx[k], startIdx[k+1]) go to device k mod (device count); as
// the reference does (one std::thread per GPU, AAPM_script/
// MultiSlicesProjGPU.cu:474-484, MultiSlicesBackGPU.cu:335-347) each device's
// slabs run on a host thread of their own, so devices work at the same time.
// DDFAN_SLAB_THREADS=slab gives every slab its own thread (several on one
// device: the library is thread-safe per plan and stream).
static int mex_call(bool forward, float x0, float y0, int DNU, const float* xds, const float* yds,
                    float detCntIdx, float imgXCenter, float imgYCenter, const float* hangs, int PN,
                    int XN, int YN, int SLN, const float* in, float dx, const uint8_t* mask,
                    const int32_t* startIdx, int nStartIdx, int sat_mode, int back_mode, float* out) {
  if (!xds || !yds || !hangs || !in || !out) return set_err(DDFAN_ERR_ARG, "null argument");
  if (PN < 1 || SLN < 1 || XN < 1 || YN < 1 || DNU < 2) return set_err(DDFAN_ERR_ARG, "bad sizes");
  std::vector<std::pair<int, int>> slabs;
  int rc = slabs_of(startIdx, nStartIdx, SLN, slabs);
  if (rc) return rc;
  const int ndev = device_count();
  if (ndev < 1) return set_err(DDFAN_ERR_CUDA, "no CUDA device");
  const size_t npix = (size_t)XN * YN, nray = (size_t)PN * DNU;
  auto run_slab = [&](size_t k) -> int {
    const int a = slabs[k].first, b = slabs[k].second, n = b - a;
    PlanDesc d{x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, XN, YN, dx, mask, n, PN,
               sat_mode, (int)(k % ndev)};
    if (n == SLN) return mex_slab(forward, d, hangs, PN, in, out, back_mode);
    std::vector<float> sin, sang, sout(forward ? nray * n : npix * n);
    gather_slab(in, forward ? npix : nray, SLN, a, b, sin);
    gather_slab(hangs, PN, SLN, a, b, sang);
    const int r = mex_slab(forward, d, sang.data(), PN, sin.data(), sout.data(), back_mode);
    if (!r) scatter_slab(sout, forward ? nray : npix, SLN, a, b, out);  // disjoint slices of out
    return r;
  };
  // slab groups: per device, or per slab
  const char* ev = getenv("DDFAN_SLAB_THREADS");
  const bool per_slab = ev && !std::strcmp(ev, "slab");
  std::vector<std::vector<size_t>> groups;
  if (per_slab) {
    for (size_t k = 0; k < slabs.size(); ++k) groups.push_back({k});
  } else {
    groups.resize(std::min<size_t>(slabs.size(), (size_t)ndev));
    for (size_t k = 0; k < slabs.size(); ++k) groups[k % ndev].push_back(k);
  }
  if (groups.size() == 1) {
    for (size_t k : groups[0])
      if ((rc = run_slab(k))) return rc;
    return DDFAN_OK;
  }
  // errors are per thread (ddfan_last_error is thread-local): carry them back
  std::vector<int> rcs(groups.size(), DDFAN_OK);
  std::vector<std::string> msgs(groups.size());
  std::vector<std::thread> threads;
  for (size_t g = 0; g < groups.size(); ++g)
    threads.emplace_back([&, g] {
      for (size_t k : groups[g]) {
        const int r = run_slab(k);
        if (r) {
          rcs[g] = r;
          msgs[g] = last_error();
          return;
        }
      }
    });
  for (std::thread& t : threads) t.join();
  for (size_t g = 0; g < groups.size(); ++g)
    if (rcs[g]) return set_err(rcs[g], "%s", msgs[g].c_str());
  return DDFAN_OK;
}

// ====================================================================== solver


static void solver_free(Solver* s) {
  if (!s) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  // release after the solver's last use (possibly on a caller's stream),
  // without synchronising the rest of the device
  if (s->own && s->last_use) {
    cudaStreamWaitEvent(s->own, s->last_use, 0);
    cudaStreamSynchronize(s->own);
  }
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->graph) cudaGraphDestroy(s->graph);
  void* ptrs[] = {s->d_vg, s->d_fc, s->d_cvd, s->d_yview, s->d_order, s->d_counts, s->d_rows, s->d_cols,
                  s->d_y, s->d_x, s->d_xprev, s->d_ax, s->d_t, s->d_perm, s->d_inv, s->d_soff, s->d_ztd,
                  s->d_xu, s->d_stage, s->d_pang, s->d_xt, s->d_tabx, s->d_taby, s->d_sq, s->d_x0};
  for (void* q : ptrs) dev_free(q, s->own);
  if (s->own) cudaStreamDestroy(s->own);
  if (s->last_use) cudaEventDestroy(s->last_use);
  cudaGetLastError();
  plan_free(s->P);
  if (prev >= 0) cudaSetDevice(prev);
  delete s;
}

template <class T>
static int salloc(Solver& s, T** p, size_t n) {
  const int rc = dev_alloc((void**)p, std::max<size_t>(n, 1) * sizeof(T), s.own);
  if (!rc) s.bytes += std::max<size_t>(n, 1) * sizeof(T);
  return rc;
}

// The internal image and sinogram use another slice order or count than the
// caller's (windowed solver; direct mode with slices padded to a multiple of 4).
static bool remapped(const Solver& s) { return s.win || (s.direct && s.Zi != s.Z); }
// The image callers read lives in d_xu (published after iterations), not d_x.
static bool published_copy(const Solver& s) {
  return s.win || s.ps || (s.direct && (s.Zi != s.Z || s.P->has_mask));
}

// Slice gathers between the caller's slice order and the internal one:
// dst[r][t] = map[t] >= 0 ? src[r][map[t]] : 0 for r < rows, t < Zd.
static __global__ void k_gather_slices(const float* __restrict__ src, int Zs, float* __restrict__ dst, int Zd,
                                       const int* __restrict__ map, size_t rows) {
  const size_t n = rows * Zd;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / Zd;
    const int t = (int)(i - r * Zd);
    const int m = map[t];
    dst[i] = m >= 0 ? src[r * Zs + m] : 0.f;
  }
}

static int gather_slices(const float* src, int Zs, float* dst, int Zd, const int* map, size_t rows,
                         cudaStream_t st) {
  const size_t n = rows * Zd;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_gather_slices<<<std::max(blocks, 1), 256, 0, st>>>(src, Zs, dst, Zd, map, rows);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "slice gather: %s", cudaGetErrorString(e));
  return DDFAN_OK;
}

// ------------------------------------------------------------ slice-major path

// Both image tables of the current image (rows from d_x, columns from its transpose).
static int ps_sat_image(Solver& s, cudaStream_t st) {
  const Plan& p = *s.P;
  int rc;
  if ((rc = ps_transpose(s.d_x, s.d_xt, s.Z, s.YN, s.XN, st))) return rc;
  PsScanArgs a{};
  a.mask = p.has_mask ? p.d_mask : nullptr;
  a.XN = s.XN;
  a.pad = 1;  // guard cells: one before the line, one after (the total)
  a.tab = s.d_tabx; a.nlines = s.Z * s.YN; a.N = s.XN; a.Nw = s.XN + 2; a.src = s.d_x; a.lines_per_slice = s.YN;
  a.cols = 0;
  if ((rc = ps_scan(p.mode, 0, a, st))) return rc;
  a.tab = s.d_taby; a.nlines = s.Z * s.XN; a.N = s.YN; a.Nw = s.YN + 2; a.src = s.d_xt; a.lines_per_slice = s.XN;
  a.cols = 1;
  return ps_scan(p.mode, 0, a, st);
}

// Subset k of a slice-major iteration: every slice's own views k, k + nOS, ...
static int ps_subset(Solver& s, int k, cudaStream_t st) {
  const Plan& p = *s.P;
  const int Z = s.Z, U = s.U, c = s.cnt[k];
  const size_t rows = (size_t)Z * s.cstride;
  int rc;
  // geometry of every slice's views of the subset
  if ((rc = launch_view_geom(p, s.d_pang + (size_t)k * rows, 1, (int)rows, s.d_vg, s.d_fc, s.d_cvd, st)))
    return rc;
  // project the current image (AAPM_script/OSSART_AAPM.m:85)
  {
    ProfScope ps(KIND_SAT_IMAGE, st);
    if ((rc = ps_sat_image(s, st))) return rc;
  }
  {
    PsFwdArgs f;
    f.tabx = s.d_tabx; f.taby = s.d_taby;
    f.vg = s.d_vg; f.fc = s.d_fc; f.cvd = s.d_cvd; f.out = s.d_ax;
    f.cstride = s.cstride; f.U = U; f.XN = s.XN; f.YN = s.YN; f.dx = (float)p.dx;
    if ((rc = ps_fwd(p.mode, f, c, Z, st))) return rc;
  }
  // residual (y - A x) / rowSum, weighted, into channel prefix sums (:86-88)
  {
    ProfScope ps(KIND_SAT_SINO, st);
    PsScanArgs r{};
    r.tab = s.d_sq; r.nlines = Z * c; r.N = U; r.Nw = U + 1;
    r.y = s.d_y; r.ax = s.d_ax; r.rows = s.d_rows; r.wgt = s.back_mode == DDFAN_BACK_ADJ ? s.d_cvd : nullptr;
    r.wscale = 1.f;
    r.cnt = c; r.cstride = s.cstride; r.P = s.PNall; r.roff = s.off[k]; r.ksub = k; r.nOS = s.nsub;
    if ((rc = ps_scan(p.mode, 1, r, st))) return rc;
  }
  // backprojection, divide by colSum, add, optional clamp (:91-97)
  PsBackArgs b{};
  b.sq = s.d_sq; b.vg = s.d_vg; b.fc = s.d_fc;
  b.tb = p.d_tb; b.lut = p.d_lut; b.t0 = p.t0; b.invdt = p.invdt; b.dirt = p.dirt; b.M = p.M;
  b.cnt = c; b.cstride = s.cstride; b.U = U; b.XN = s.XN; b.YN = s.YN;
  b.ocx = p.ocx; b.ocy = p.ocy; b.dx = p.dx;
  b.inv_sid = p.inv_sid; b.inv_dbeta = p.inv_dbeta; b.cnt_ref = (double)p.detCntIdx + 0.5;
  b.x = s.d_x; b.colsum = s.d_cols + (size_t)k * s.XN * s.YN; b.nonneg = s.nonneg;
  b.mask = p.has_mask ? p.d_mask : nullptr;
  return s.back_mode == DDFAN_BACK_ADJ ? ps_back(p.mode, b, Z, st) : ps_back_ref(p.mode, b, Z, st);
}

// One OS-SART iteration (AAPM_script/OSSART_AAPM.m:79-115) on stream st.
static int solver_iteration(Solver& s, cudaStream_t st) {
  Plan& p = *s.P;
  int rc, n = 0;
  const bool adj = s.back_mode == DDFAN_BACK_ADJ;
  for (int k = 0; k < s.nsub && s.ps; ++k) {
    if ((rc = ps_subset(s, k, st))) return rc;
    n += 7;
  }
  for (int k = 0; k < s.nsub && s.direct; ++k) {
    const int o = s.off[k], c = s.cnt[k];
    BackEpi e{};
    e.out = s.d_x; e.xin = s.d_x; e.colsum = s.d_cols + (size_t)k * s.XN * s.YN;
    e.nonneg = s.nonneg; e.mask = p.has_mask ? p.d_mask : nullptr; e.zlo = 0; e.zhi = s.Zi;
    const ViewGeom* vg = s.d_vg + o;
    const double2* fc = s.d_fc + (size_t)o * (s.U + 1);
    const float* cvd = s.d_cvd + (size_t)o * s.U;
    // project the current image and store the residual (y - A x) / rowSum,
    // weighted for the exact adjoint (AAPM_script/OSSART_AAPM.m:85-88)
    DdResidual r;
    r.y = s.d_y; r.yview = s.d_yview + o; r.rowsum = s.d_rows + (size_t)o * s.U; r.wgt = adj ? cvd : nullptr;
    r.ystride = s.Zi;
    if ((rc = launch_fwd_dd(p, s.d_x, vg, fc, cvd, s.d_order + o, c, s.d_ax, s.U + 1, s.Zi, 0, s.Zi, &r, st)))
      return rc;
    // backproject, divide by colSum, add, optional clamp (:91-97)
    if ((rc = launch_back_dd(p, s.back_mode, s.d_ax, vg, fc, s.d_order + o, s.d_counts + 2 * k, c, e, st)))
      return rc;
    n += adj ? 3 : 2;
  }
  for (int k = 0; k < s.nsub && !s.ps && !s.direct; ++k) {
    const int o = s.off[k], c = s.cnt[k];
    BackEpi e{};
    e.out = s.d_x; e.xin = s.d_x; e.colsum = s.d_cols + (size_t)k * s.XN * s.YN;
    e.nonneg = s.nonneg; e.mask = p.has_mask ? p.d_mask : nullptr; e.zlo = 0; e.zhi = s.Zi;
    // project the current image (:85)
    if ((rc = launch_sat_image(p, s.d_x, st))) return rc;
    if (!s.win) {
      const ViewGeom* vg = s.d_vg + o;
      const double2* fc = s.d_fc + (size_t)o * (s.U + 1);
      const float* cvd = s.d_cvd + (size_t)o * s.U;
      if ((rc = launch_fwd(p, vg, fc, cvd, s.d_order + o, c, s.d_ax, 0, s.Zi, st))) return rc;
      // residual (y - A x) / rowSum folded into the sinogram prefix sums (:86-88)
      if ((rc = launch_sat_sino(p, s.d_ax, c, adj ? cvd : nullptr, 1.f, s.d_y, s.d_yview + o,
                                s.d_rows + (size_t)o * s.U, st)))
        return rc;
      // backproject, divide by colSum, add, optional clamp (:91-97)
      if ((rc = launch_back(p, s.back_mode, vg, fc, s.d_order + o, s.d_counts + 2 * k, c, e, st))) return rc;
    } else {
      const int4* ztd = s.d_ztd + (size_t)k * s.nzt;
      const int m = s.maxcnt[k];
      ViewRanges vr;
      vr.ztd = ztd; vr.soff = s.d_soff; vr.Mc = s.Mc; vr.nOS = s.nsub; vr.ksub = k; vr.T = s.PNall;
      if ((rc = launch_fwd(p, s.d_vg, s.d_fc, s.d_cvd, s.d_order, m, s.d_ax, 0, s.Zi, st, ztd))) return rc;
      if ((rc = launch_sat_sino(p, s.d_ax, m, adj ? s.d_cvd : nullptr, 1.f, s.d_y, nullptr,
                                s.d_rows + (size_t)o * s.U, st, 0, s.Zi, &vr)))
        return rc;
      if ((rc = launch_back(p, s.back_mode, s.d_vg, s.d_fc, s.d_order, nullptr, m, e, st, ztd))) return rc;
    }
    n += adj ? 5 : 4;
  }
  if (s.useFISTA) {
    const size_t V = (size_t)s.XN * s.YN * s.Zi;
    const int blocks = (int)std::min<size_t>((V + 255) / 256, 148 * 16);
    ProfScope ps(KIND_FISTA, st);
    k_fista<<<blocks, 256, 0, st>>>(s.d_x, s.d_xprev, V, s.d_t);
    k_fista_t<<<1, 1, 0, st>>>(s.d_t);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "fista launch: %s", cudaGetErrorString(e));
    n += 2;
  }
  s.launches = n;
  return DDFAN_OK;
}

// The image in the caller's layout and slice order (windowed and slice-major
// solvers), after iterations.
static int solver_publish(Solver& s, cudaStream_t st) {
  if (s.ps) return ps_transpose(s.d_x, s.d_xu, 1, s.Z, s.XN * s.YN, st);
  if (s.direct && s.P->has_mask)
    return launch_publish_masked(s.d_x, s.Zi, s.d_x0, s.Z, s.P->d_mask, s.nonneg && s.iters_done > 0 ? 1 : 0,
                                 s.d_xu, (size_t)s.XN * s.YN, st);
  if (!remapped(s)) return DDFAN_OK;
  return gather_slices(s.d_x, s.Zi, s.d_xu, s.Z, s.d_inv, (size_t)s.XN * s.YN, st);
}

int solver_after_iterations(Solver& s, int n, cudaStream_t st) {
  s.iters_done += n;
  int rc = solver_publish(s, st);
  if (!rc) cudaEventRecord(s.last_use, st);
  return rc;
}

// Every slice's angle list as a window of one raw-view table: view ib of
// slice z is G[off[z] + ib], bitwise.  A slice continues the table where its
// list overlaps the previous slice's window end (helical rebinning: slice z+1
// starts a few raw views after slice z), reuses an identical earlier window,
// or appends its whole list.
static void angle_windows(const float* hangs, int T, int SLN, std::vector<float>& G, std::vector<int>& off) {
  G.clear();
  off.assign(SLN, 0);
  auto bits = [](float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; };
  auto at = [&](int ib, int z) { return bits(hangs[(size_t)ib * SLN + z]); };
  std::unordered_map<uint64_t, std::vector<int>> seen;  // list hash -> slices with that window
  for (int z = 0; z < SLN; ++z) {
    uint64_t h = 1469598103934665603ull;
    for (int ib = 0; ib < T; ++ib) h = (h ^ at(ib, z)) * 1099511628211ull;
    int placed = -1;
    if (z > 0 && (size_t)off[z - 1] + T == G.size()) {
      const int base = off[z - 1];
      const uint32_t first = at(0, z);
      for (int d = 0; d < T && placed < 0; ++d) {
        if (bits(G[base + d]) != first) continue;
        bool ok = true;
        for (int ib = 0; ib < T - d && ok; ++ib) ok = at(ib, z) == bits(G[base + d + ib]);
        if (ok) {
          placed = base + d;
          for (int ib = T - d; ib < T; ++ib) G.push_back(hangs[(size_t)ib * SLN + z]);
        }
      }
    }
    if (placed < 0) {
      for (int y : seen[h]) {
        bool ok = true;
        for (int ib = 0; ib < T && ok; ++ib) ok = at(ib, z) == at(ib, y);
        if (ok) {
          placed = off[y];
          break;
        }
      }
    }
    if (placed < 0) {
      placed = (int)G.size();
      for (int ib = 0; ib < T; ++ib) G.push_back(hangs[(size_t)ib * SLN + z]);
    }
    off[z] = placed;
    seen[h].push_back(z);
  }
}

// Internal slice order, z-tile width and view ranges of the windowed solver.
struct WinLayout {
  int ZL = 1, Zi = 0, nzt = 0, Mc = 1, PNmax = 0;
  std::vector<int> perm, soff;
  std::vector<int4> ztd;  // [nsub][nzt], .w filled on the device
  std::vector<int> maxcnt;
  long long cost = 0;
};

static void win_layout(const std::vector<int>& off, int NG, int T, int nOS, int ZL, WinLayout& w) {
  const int SLN = (int)off.size();
  w.ZL = ZL;
  w.Mc = (NG + nOS - 1) / nOS + 1;
  std::vector<int> idx(SLN);
  for (int z = 0; z < SLN; ++z) idx[z] = z;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
    const int ra = off[a] % nOS, rb = off[b] % nOS;
    return ra != rb ? ra < rb : off[a] < off[b];
  });
  const int tile = 4 * ZL;
  w.perm.clear();
  for (size_t i = 0; i < idx.size();) {
    size_t j = i;
    const int r = off[idx[i]] % nOS;
    while (j < idx.size() && off[idx[j]] % nOS == r) w.perm.push_back(idx[j++]);
    while (w.perm.size() % tile) w.perm.push_back(-1);
    i = j;
  }
  w.Zi = (int)w.perm.size();
  w.nzt = w.Zi / tile;
  w.soff.assign(w.Zi, INT_MAX);
  for (int t = 0; t < w.Zi; ++t)
    if (w.perm[t] >= 0) w.soff[t] = off[w.perm[t]];
  w.ztd.assign((size_t)nOS * w.nzt, make_int4(0, 0, 0, 0));
  w.maxcnt.assign(nOS, 0);
  w.PNmax = 0;
  w.cost = 0;
  int ooff = 0;
  for (int k = 0; k < nOS; ++k) {
    for (int zt = 0; zt < w.nzt; ++zt) {
      int lo = INT_MAX, hi = INT_MIN, r = 0;
      for (int t = zt * tile; t < (zt + 1) * tile; ++t)
        if (w.perm[t] >= 0) {
          lo = std::min(lo, w.soff[t]);
          hi = std::max(hi, w.soff[t] + T - 1);
          r = w.soff[t] % nOS;
        }
      const int c = (r + k) % nOS;
      // raw views g = c (mod nOS) in [lo, hi]
      const int gf = lo + ((c - lo % nOS) % nOS + nOS) % nOS;
      const int count = gf > hi ? 0 : (hi - gf) / nOS + 1;
      w.ztd[(size_t)k * w.nzt + zt] = make_int4(c * w.Mc + (gf - c) / nOS, count, ooff, 0);
      ooff += count;
      w.maxcnt[k] = std::max(w.maxcnt[k], count);
      w.PNmax = std::max(w.PNmax, count);
      w.cost += (long long)count;
    }
  }
}

// Row sums and column sums of every subset from slice 0's angles, on a
// one-slice plan (AAPM_script/OSSART_AAPM.m:57-66), with the 4-slice cell
// kernels: the REF backprojector's weights, and the exact adjoint's for more
// than 65535 geometry rows.
// The row sums of all views go in one forward launch; the column sums one
// subset at a time on the solver's stream (spreading them over side streams
// cut a lone solver's set-up by 5 ms but cost batched solves 20 % of their
// throughput, as those latency-bound one-slice launches took SM slots from
// the other solves).
static int solver_weights_cells(Solver& s, const PlanDesc& d, const std::vector<float>& angs0, int PNmax,
                                cudaStream_t st) {
  const int XN = s.XN, YN = s.YN, DNU = s.U, P = s.PNall;
  PlanDesc d1 = d;
  d1.SLN = 1;
  d1.PNmax = PNmax;
  d1.zl_force = 0;
  d1.sat_mode = cell_mode(d.sat_mode);
  PlanPtr P1;
  int rc = plan_create(&P1.p, d1);
  if (rc) return rc;
  DevBuf<ViewGeom> vg(st);
  DevBuf<double2> fc(st);
  DevBuf<float> cvd(st), ang(st), ones(st);
  DevBuf<int> order(st), counts(st), order_all(st), counts_all(st);
  const size_t n1 = std::max((size_t)XN * YN, (size_t)PNmax * DNU);
  if ((rc = vg.alloc(P)) || (rc = fc.alloc((size_t)P * (DNU + 1))) || (rc = cvd.alloc((size_t)P * DNU)) ||
      (rc = ang.alloc(P)) || (rc = ones.alloc(n1)) || (rc = order.alloc(P)) || (rc = counts.alloc(2 * (size_t)s.nsub)) ||
      (rc = order_all.alloc(P)) || (rc = counts_all.alloc(2)))
    return rc;
  std::vector<float> h1(n1, 1.0f);
  DDFAN_CK(cudaMemcpyAsync(ones.p, h1.data(), sizeof(float) * n1, cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemcpyAsync(ang.p, angs0.data(), sizeof(float) * P, cudaMemcpyHostToDevice, st));
  if ((rc = launch_view_geom(*P1.p, ang.p, 1, P, vg.p, fc.p, cvd.p, st))) return rc;
  for (int k = 0; k < s.nsub; ++k)
    if ((rc = launch_view_order(vg.p + s.off[k], s.cnt[k], order.p + s.off[k], counts.p + 2 * k, st))) return rc;
  if ((rc = launch_view_order(vg.p, P, order_all.p, counts_all.p, st))) return rc;
  if ((rc = launch_sat_image(*P1.p, ones.p, st))) return rc;
  if ((rc = launch_fwd(*P1.p, vg.p, fc.p, cvd.p, order_all.p, P, s.d_rows, 0, 1, st))) return rc;
  const bool adj = s.back_mode == DDFAN_BACK_ADJ;
  for (int k = 0; k < s.nsub; ++k) {
    const int o = s.off[k], c = s.cnt[k];
    if ((rc = launch_sat_sino(*P1.p, ones.p, c, adj ? cvd.p + (size_t)o * DNU : nullptr, 1.f, nullptr, nullptr,
                              nullptr, st)))
      return rc;
    BackEpi e{};
    e.out = s.d_cols + (size_t)k * XN * YN;
    e.mask = P1.p->has_mask ? P1.p->d_mask : nullptr;
    e.zlo = 0; e.zhi = 1;
    if ((rc = launch_back(*P1.p, s.back_mode, vg.p + o, fc.p + (size_t)o * (DNU + 1), order.p + o,
                          counts.p + 2 * k, c, e, st)))
      return rc;
  }
  DDFAN_CK(cudaStreamSynchronize(st));
  return DDFAN_OK;
}

// Row sums and column sums of every subset from slice 0's angles
// (AAPM_script/OSSART_AAPM.m:57-66) on the slice-major kernels, which carry
// one slice without the 4-slice cells' padding: the row sums of all views in
// one forward launch, and the column sums of all subsets in one
// backprojection launch, subset k standing in the place of slice k (its views
// are rows k * cs + m; the pad rows of a short subset backproject zeros).
// The exact adjoint only: the slice-major REF backprojector takes its
// half-width and weight in FP32, and column sums divide every update, so the
// REF weights stay on the cell kernels' FP64 formula.
static int solver_weights(Solver& s, const PlanDesc& d, const std::vector<float>& angs0, int PNmax,
                          cudaStream_t st) {
  const int XN = s.XN, YN = s.YN, DNU = s.U, nsub = s.nsub, cs = PNmax;
  const size_t R = (size_t)nsub * cs;  // geometry rows [nsub][cs]
  const bool adj = s.back_mode == DDFAN_BACK_ADJ;
  if (R > 65535 || !adj) return solver_weights_cells(s, d, angs0, PNmax, st);
  PlanDesc d1 = d;
  d1.SLN = 1;
  d1.PNmax = 1;
  d1.zl_force = 0;
  d1.sat_mode = cell_mode(d.sat_mode);
  PlanPtr P1;
  int rc = plan_create(&P1.p, d1);
  if (rc) return rc;
  const Plan& p = *P1.p;
  if (!p.adj_ok) return set_err(DDFAN_ERR_UNSUPPORTED, "detector boundaries are not monotone as seen from the source");
  // angles [nsub][cs] and the ones to project: an image of ones and, per
  // subset, cs rows of ones over its views (zeros on pad rows)
  std::vector<float> wa(R, 0.f), himg((size_t)XN * YN, 1.f), hsino(R * DNU, 0.f);
  DevBuf<float> ang(st), img(st), ones(st), rows(st), sino(st);
  DevBuf<ViewGeom> vg(st);
  DevBuf<double2> fc(st);
  DevBuf<float> cvd(st);
  const size_t CF = p.mode == SAT_FP32 ? 2 : 4;  // floats per slice-major cell
  DevBuf<float> tabx(st), taby(st), sq(st);
  if ((rc = ang.alloc(R)) || (rc = vg.alloc(R)) || (rc = fc.alloc(R * (DNU + 1))) || (rc = cvd.alloc(R * DNU)) ||
      (rc = img.alloc((size_t)XN * YN)) || (rc = rows.alloc(R * DNU)) || (rc = sino.alloc(R * DNU)) ||
      (rc = tabx.alloc(CF * (XN + 2) * YN)) || (rc = taby.alloc(CF * (YN + 2) * XN)) ||
      (rc = sq.alloc(CF * R * (DNU + 1))))
    return rc;
  for (int k = 0; k < nsub; ++k)
    for (int m = 0; m < s.cnt[k]; ++m) wa[(size_t)k * cs + m] = angs0[(size_t)s.off[k] + m];
  DDFAN_CK(cudaMemcpyAsync(ang.p, wa.data(), sizeof(float) * R, cudaMemcpyHostToDevice, st));
  for (int k = 0; k < nsub; ++k)
    std::fill(hsino.begin() + (size_t)k * cs * DNU, hsino.begin() + ((size_t)k * cs + s.cnt[k]) * DNU, 1.f);
  DDFAN_CK(cudaMemcpyAsync(img.p, himg.data(), sizeof(float) * XN * YN, cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemcpyAsync(sino.p, hsino.data(), sizeof(float) * R * DNU, cudaMemcpyHostToDevice, st));
  if ((rc = launch_view_geom(p, ang.p, 1, (int)R, vg.p, fc.p, cvd.p, st))) return rc;
  // prefix-sum tables of the masked ones image (rows and columns: the image is its own transpose)
  PsScanArgs a{};
  a.mask = p.has_mask ? p.d_mask : nullptr;
  a.XN = XN; a.pad = 1; a.src = img.p;
  a.tab = tabx.p; a.nlines = YN; a.N = XN; a.Nw = XN + 2; a.lines_per_slice = YN;
  if ((rc = ps_scan(p.mode, 0, a, st))) return rc;
  a.tab = taby.p; a.nlines = XN; a.N = YN; a.Nw = YN + 2; a.lines_per_slice = XN; a.cols = 1;
  if ((rc = ps_scan(p.mode, 0, a, st))) return rc;
  // row sums: every view row of the one slice, then into subset order
  PsFwdArgs f;
  f.tabx = tabx.p; f.taby = taby.p; f.vg = vg.p; f.fc = fc.p; f.cvd = cvd.p;
  f.out = rows.p; f.cstride = (int)R; f.U = DNU; f.XN = XN; f.YN = YN; f.dx = (float)p.dx;
  if ((rc = ps_fwd(p.mode, f, (int)R, 1, st))) return rc;
  for (int k = 0; k < nsub; ++k)
    DDFAN_CK(cudaMemcpyAsync(s.d_rows + (size_t)s.off[k] * DNU, rows.p + (size_t)k * cs * DNU,
                             sizeof(float) * s.cnt[k] * DNU, cudaMemcpyDeviceToDevice, st));
  // column sums: subset k as slice k, weighted like the solver's residual
  PsScanArgs q{};
  q.tab = sq.p; q.nlines = (int)R; q.N = DNU; q.Nw = DNU + 1; q.src = sino.p; q.lines_per_slice = 1;
  q.wgt = cvd.p; q.wscale = 1.f;
  if ((rc = ps_scan(p.mode, 2, q, st))) return rc;
  PsBackArgs b{};
  b.sq = sq.p; b.vg = vg.p; b.fc = fc.p;
  b.tb = p.d_tb; b.lut = p.d_lut; b.t0 = p.t0; b.invdt = p.invdt; b.dirt = p.dirt; b.M = p.M;
  b.cnt = cs; b.cstride = cs; b.U = DNU; b.XN = XN; b.YN = YN;
  b.ocx = p.ocx; b.ocy = p.ocy; b.dx = p.dx;
  b.inv_sid = p.inv_sid; b.inv_dbeta = p.inv_dbeta; b.cnt_ref = (double)p.detCntIdx + 0.5;
  b.out = s.d_cols; b.mask = p.has_mask ? p.d_mask : nullptr;
  if ((rc = ps_back(p.mode, b, nsub, st))) return rc;
  // the pageable host sources above are consumed and the temporaries free after this
  DDFAN_CK(cudaStreamSynchronize(st));
  return DDFAN_OK;
}

// The windowed cost (projector work over that of shared lists) above which
// the slice-major path is faster, per backprojector.  Measured at
// 512 x 512 x 128, 24 subsets of 96 views: slice-major iterations take 2.05x
// (exact adjoint) and 2.9x (REF, FP64 geometry per sample and slice) the
// shared-list time whatever the lists; windowed ones about 1.2x their
// modelled cost (2.13x and 2.2x at a model of 1.76 for slices 36 raw views
// apart, 13.5x at 13.3 for 86.07 apart).
static constexpr double kSliceMajorCostAdj = 1.7, kSliceMajorCostRef = 2.4;

static int solver_create(Solver** out, float x0, float y0, int DNU, const float* xds, const float* yds,
                         float detCntIdx, float imgXCenter, float imgYCenter, const float* hangs,
                         int PNall, int XN, int YN, int SLN, float dx, const uint8_t* mask,
                         int numOfOS, int useFISTA, int nonneg, int sat_mode, int back_mode,
                         int device) {
  *out = nullptr;
  if (!hangs || !xds || !yds) return set_err(DDFAN_ERR_ARG, "null argument");
  if (numOfOS < 1 || numOfOS > PNall) return set_err(DDFAN_ERR_ARG, "numOfOS=%d outside [1, %d]", numOfOS, PNall);
  if (back_mode != DDFAN_BACK_REF && back_mode != DDFAN_BACK_ADJ)
    return set_err(DDFAN_ERR_ARG, "back_mode %d", back_mode);
  if (SLN < 1 || PNall < 1) return set_err(DDFAN_ERR_ARG, "SLN=%d PNall=%d", SLN, PNall);
  std::unique_ptr<Solver, void (*)(Solver*)> S(new Solver(), solver_free);
  Solver& s = *S;
  s.device = device; s.PNall = PNall; s.nsub = numOfOS; s.useFISTA = useFISTA ? 1 : 0;
  s.nonneg = nonneg ? 1 : 0; s.back_mode = back_mode; s.XN = XN; s.YN = YN; s.U = DNU; s.Z = SLN;
  // subsets k, k + numOfOS, ... (AAPM_script/OSSART_AAPM.m:60)
  std::vector<int> yview;
  int PNsub = 0;
  for (int k = 0; k < numOfOS; ++k) {
    s.off.push_back((int)yview.size());
    for (int v = k; v < PNall; v += numOfOS) yview.push_back(v);
    s.cnt.push_back((int)yview.size() - s.off.back());
    PNsub = std::max(PNsub, s.cnt.back());
  }
  const size_t P = (size_t)PNall;
  std::vector<float> angs0(P);  // slice 0's angles, subset order
  for (size_t r = 0; r < P; ++r) angs0[r] = hangs[(size_t)yview[r] * SLN];
  // per-slice angle lists as windows of one raw-view table
  std::vector<float> G;
  std::vector<int> woff;
  angle_windows(hangs, PNall, SLN, G, woff);
  s.win = false;
  for (int z = 1; z < SLN; ++z) s.win = s.win || woff[z] != woff[0];
  WinLayout W;
  double win_cost = 0.0;  // windowed projector work relative to shared angle lists
  if (s.win) {
    // z-tile width: views per tile x blocks per tile x relative cost of a block
    // at that width (the projector cost model of pow2_zl)
    const int widths[4] = {1, 2, 4, 8};
    const double unit[4] = {3.6, 2.1, 1.2, 1.0};
    double best = -1;
    for (int i = 0; i < 4; ++i) {
      WinLayout t;
      win_layout(woff, (int)G.size(), PNall, numOfOS, widths[i], t);
      const double c = (double)t.cost * widths[i] * unit[i];
      if (best < 0 || c < best) {
        best = c;
        W = t;
      }
    }
    win_cost = best / ((double)PNall * ((SLN + 3) / 4));
  }
  // Per-slice angle lists whose windows share little go to the slice-major
  // path, whose cost relative to shared lists does not depend on the lists; DDFAN_PER_SLICE=windowed or =slices overrides the
  // choice (=slices also for shared lists).
  {
    const char* pv = getenv("DDFAN_PER_SLICE");
    const bool want_win = pv && !std::strcmp(pv, "windowed");
    const bool want_ps = pv && !std::strcmp(pv, "slices");
    const double threshold = back_mode == DDFAN_BACK_ADJ ? kSliceMajorCostAdj : kSliceMajorCostRef;
    s.ps = want_ps || (s.win && !want_win && win_cost > threshold);
    if (s.ps) s.win = false;
  }
  // the direct mode serves one angle list for all slices; the per-slice
  // paths keep hi/lo tables
  s.direct = sat_mode == SAT_DIRECT && !s.win && !s.ps;
  if (sat_mode == SAT_DIRECT && !s.direct) sat_mode = cell_mode(sat_mode);
  if (s.win) {
    s.Zi = W.Zi; s.nzt = W.nzt; s.Mc = W.Mc; s.perm = W.perm; s.maxcnt = W.maxcnt;
  } else if (s.direct) {
    s.Zi = (SLN + 3) / 4 * 4;
    s.perm.assign(s.Zi, -1);
    for (int z = 0; z < SLN; ++z) s.perm[z] = z;
  } else {
    s.Zi = SLN;
  }
  const int PNmax = s.win ? W.PNmax : PNsub;
  PlanDesc d{x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, XN, YN, dx, mask, s.Zi, std::max(PNmax, 1),
             sat_mode, device};
  if (s.win) d.zl_force = W.ZL;
  // the slice-major path uses the plan's geometry, mask and bracket tables only
  PlanDesc dp = d;
  if (s.ps) dp.SLN = dp.PNmax = 1;
  int rc = plan_create(&s.P, dp);
  if (rc) return rc;
  s.bytes = s.P->bytes;
  DeviceGuard g(device);
  const size_t V = (size_t)XN * YN * s.Zi;
  if (s.ps) s.cstride = PNsub;
  const size_t R = s.win ? (size_t)numOfOS * s.Mc : (s.ps ? (size_t)SLN * s.cstride : P);  // geometry rows
  const size_t nord = s.win ? (size_t)std::max<long long>(W.cost, 1) : (s.ps ? 1 : P);
  DDFAN_CK(cudaStreamCreateWithFlags(&s.own, cudaStreamNonBlocking));
  DDFAN_CK(cudaEventCreateWithFlags(&s.last_use, cudaEventDisableTiming));
  if ((rc = salloc(s, &s.d_vg, R)) || (rc = salloc(s, &s.d_fc, R * (DNU + 1))) ||
      (rc = salloc(s, &s.d_cvd, R * DNU)) || (rc = salloc(s, &s.d_yview, P)) || (rc = salloc(s, &s.d_order, nord)) ||
      (rc = salloc(s, &s.d_counts, 2 * (size_t)numOfOS)) || (rc = salloc(s, &s.d_rows, P * DNU)) ||
      (rc = salloc(s, &s.d_cols, (size_t)numOfOS * XN * YN)) || (rc = salloc(s, &s.d_y, P * DNU * s.Zi)) ||
      (rc = salloc(s, &s.d_x, V)) || (rc = salloc(s, &s.d_xprev, V)) ||
      (rc = salloc(s, &s.d_ax, (size_t)std::max(PNmax, 1) * (DNU + (s.direct ? 1 : 0)) * s.Zi)) ||
      (rc = salloc(s, &s.d_t, 1)))
    return rc;
  cudaStream_t st = s.own;
  if (s.direct) {
    // the residual's guard channel stays 0; slice maps for padded slices; the
    // initial image where masked voxels keep it
    DDFAN_CK(cudaMemsetAsync(s.d_ax, 0, sizeof(float) * (size_t)std::max(PNmax, 1) * (DNU + 1) * s.Zi, st));
    const size_t Vc = (size_t)XN * YN * SLN;
    if (s.Zi != SLN) {
      std::vector<int> inv(SLN);
      for (int z = 0; z < SLN; ++z) inv[z] = z;
      if ((rc = salloc(s, &s.d_perm, s.Zi)) || (rc = salloc(s, &s.d_inv, SLN)) ||
          (rc = salloc(s, &s.d_stage, P * DNU * SLN)))
        return rc;
      DDFAN_CK(cudaMemcpyAsync(s.d_perm, s.perm.data(), sizeof(int) * s.Zi, cudaMemcpyHostToDevice, st));
      DDFAN_CK(cudaMemcpyAsync(s.d_inv, inv.data(), sizeof(int) * SLN, cudaMemcpyHostToDevice, st));
    }
    if (s.P->has_mask && (rc = salloc(s, &s.d_x0, Vc))) return rc;
    if (published_copy(s) && (rc = salloc(s, &s.d_xu, Vc))) return rc;
    DDFAN_CK(cudaStreamSynchronize(st));
  }
  DDFAN_CK(cudaMemcpyAsync(s.d_yview, yview.data(), sizeof(int) * P, cudaMemcpyHostToDevice, st));
  if (s.ps) {
    // angles of view k + m * numOfOS of every slice z, per subset k: row (k, z, m)
    std::vector<float> pang((size_t)numOfOS * SLN * s.cstride, 0.f);
    for (int k = 0; k < numOfOS; ++k)
      for (int z = 0; z < SLN; ++z)
        for (int m = 0; m < s.cnt[k]; ++m)
          pang[((size_t)k * SLN + z) * s.cstride + m] = hangs[(size_t)(k + m * numOfOS) * SLN + z];
    const size_t CF = sat_mode == SAT_FP32 ? 2 : 4;  // floats per slice-major cell
    const size_t VG = (size_t)(XN + 2) * (YN + 2) * SLN;  // cells of a table with guard cells
    if ((rc = salloc(s, &s.d_pang, pang.size())) || (rc = salloc(s, &s.d_xt, V)) ||
        (rc = salloc(s, &s.d_tabx, CF * VG)) || (rc = salloc(s, &s.d_taby, CF * VG)) ||
        (rc = salloc(s, &s.d_sq, CF * R * (DNU + 1))) || (rc = salloc(s, &s.d_xu, V)) ||
        (rc = salloc(s, &s.d_stage, P * DNU * SLN)))
      return rc;
    DDFAN_CK(cudaMemcpyAsync(s.d_pang, pang.data(), sizeof(float) * pang.size(), cudaMemcpyHostToDevice, st));
    DDFAN_CK(cudaStreamSynchronize(st));
  } else if (!s.win) {
    // per-view tables for every view, in subset order; per subset the views
    // of one orientation together (one image table at a time stays hot in
    // L2; the exact adjoint visits each orientation in turn)
    DevBuf<float> dang(st);
    if ((rc = dang.alloc(P))) return rc;
    DDFAN_CK(cudaMemcpyAsync(dang.p, angs0.data(), sizeof(float) * P, cudaMemcpyHostToDevice, st));
    if ((rc = launch_view_geom(*s.P, dang.p, 1, PNall, s.d_vg, s.d_fc, s.d_cvd, st))) return rc;
    for (int k = 0; k < numOfOS; ++k)
      if ((rc = launch_view_order(s.d_vg + s.off[k], s.cnt[k], s.d_order + s.off[k], s.d_counts + 2 * k, st)))
        return rc;
    DDFAN_CK(cudaStreamSynchronize(st));
  } else {
    // raw-view geometry rows, grouped by residue; per (subset, z-tile) range
    // the slot order (x-major first) and its x-major count
    std::vector<float> rows(R, 0.f), soff_h(W.soff.begin(), W.soff.end());
    for (size_t r = 0; r < R; ++r) {
      const size_t gv = r / s.Mc + (r % s.Mc) * (size_t)numOfOS;
      if (gv < G.size()) rows[r] = G[gv];
    }
    std::vector<int> inv(SLN, 0);
    for (int t = 0; t < s.Zi; ++t)
      if (s.perm[t] >= 0) inv[s.perm[t]] = t;
    DevBuf<float> dang(st);
    if ((rc = dang.alloc(R)) || (rc = salloc(s, &s.d_perm, s.Zi)) || (rc = salloc(s, &s.d_inv, SLN)) ||
        (rc = salloc(s, &s.d_soff, s.Zi)) || (rc = salloc(s, &s.d_ztd, W.ztd.size())) ||
        (rc = salloc(s, &s.d_xu, (size_t)XN * YN * SLN)) || (rc = salloc(s, &s.d_stage, P * DNU * SLN)))
      return rc;
    DDFAN_CK(cudaMemcpyAsync(dang.p, rows.data(), sizeof(float) * R, cudaMemcpyHostToDevice, st));
    DDFAN_CK(cudaMemcpyAsync(s.d_perm, s.perm.data(), sizeof(int) * s.Zi, cudaMemcpyHostToDevice, st));
    DDFAN_CK(cudaMemcpyAsync(s.d_inv, inv.data(), sizeof(int) * SLN, cudaMemcpyHostToDevice, st));
    DDFAN_CK(cudaMemcpyAsync(s.d_soff, W.soff.data(), sizeof(int) * s.Zi, cudaMemcpyHostToDevice, st));
    DDFAN_CK(cudaMemcpyAsync(s.d_ztd, W.ztd.data(), sizeof(int4) * W.ztd.size(), cudaMemcpyHostToDevice, st));
    if ((rc = launch_view_geom(*s.P, dang.p, 1, (int)R, s.d_vg, s.d_fc, s.d_cvd, st))) return rc;
    if ((rc = launch_view_order_ranges(s.d_vg, s.d_ztd, (int)W.ztd.size(), s.d_order, st))) return rc;
    DDFAN_CK(cudaMemsetAsync(s.d_xu, 0, sizeof(float) * XN * YN * SLN, st));
    DDFAN_CK(cudaStreamSynchronize(st));
  }
  if ((rc = solver_weights(s, d, angs0, PNsub, st))) return rc;
  const double one = 1.0;
  DDFAN_CK(cudaMemcpyAsync(s.d_t, &one, sizeof(double), cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemsetAsync(s.d_x, 0, sizeof(float) * V, st));
  DDFAN_CK(cudaMemsetAsync(s.d_xprev, 0, sizeof(float) * V, st));
  DDFAN_CK(cudaMemsetAsync(s.d_y, 0, sizeof(float) * P * DNU * s.Zi, st));
  DDFAN_CK(cudaStreamSynchronize(st));
  *out = S.release();
  return DDFAN_OK;
}

}  // namespace ddfan

using namespace ddfan;

extern "C" {

DDFAN_API int ddfan_MultiSlicesProjGPU(float x0, float y0, int DNU, const float* xds, const float* yds,
                                       float imgXCenter, float imgYCenter, const float* hangs, int PN,
                                       int XN, int YN, int SLN, const float* vol, float dx,
                                       const uint8_t* mask, const int32_t* startIdx, int nStartIdx,
                                       int sat_mode, float* prj) {
  return mex_call(true, x0, y0, DNU, xds, yds, 0.f, imgXCenter, imgYCenter, hangs, PN, XN, YN, SLN,
                  vol, dx, mask, startIdx, nStartIdx, sat_mode, DDFAN_BACK_REF, prj);
}

DDFAN_API int ddfan_MultiSlicesBackGPU(float x0, float y0, int DNU, const float* xds, const float* yds,
                                       float detCntIdx, float imgXCenter, float imgYCenter,
                                       const float* hangs, int PN, int XN, int YN, int SLN,
                                       const float* prj, float dx, const uint8_t* mask,
                                       const int32_t* startIdx, int nStartIdx, int sat_mode,
                                       int back_mode, float* vol) {
  if (back_mode != DDFAN_BACK_REF && back_mode != DDFAN_BACK_ADJ)
    return set_err(DDFAN_ERR_ARG, "back_mode %d", back_mode);
  return mex_call(false, x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PN, XN, YN,
                  SLN, prj, dx, mask, startIdx, nStartIdx, sat_mode, back_mode, vol);
}

DDFAN_API int ddfan_ossart_create(ddfan_ossart** out, float x0, float y0, int DNU, const float* xds,
                                  const float* yds, float detCntIdx, float imgXCenter, float imgYCenter,
                                  const float* hangs, int PNall, int XN, int YN, int SLN, float dx,
                                  const uint8_t* mask, int numOfOS, int useFISTA, int nonneg,
                                  int sat_mode, int back_mode, int device) {
  if (!out) return set_err(DDFAN_ERR_ARG, "out is null");
  Solver* s = nullptr;
  int rc = solver_create(&s, x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PNall,
                         XN, YN, SLN, dx, mask, numOfOS, useFISTA, nonneg, sat_mode, back_mode, device);
  *out = reinterpret_cast<ddfan_ossart*>(s);
  return rc;
}

DDFAN_API void ddfan_ossart_destroy(ddfan_ossart* s) { solver_free(reinterpret_cast<Solver*>(s)); }

DDFAN_API size_t ddfan_ossart_estimate_bytes(int XN, int YN, int DNU, int SLN, int PNall, int numOfOS,
                                             int sat_mode) {
  if (numOfOS < 1 || PNall < numOfOS) return 0;
  const size_t PNmax = (size_t)(PNall + numOfOS - 1) / numOfOS;
  const bool direct = sat_mode == SAT_DIRECT;
  // the direct mode pads slices to a multiple of 4 and keeps a guard channel
  const size_t Zi = direct ? (size_t)(SLN + 3) / 4 * 4 : (size_t)SLN;
  const size_t U = (size_t)DNU, P = (size_t)PNall, V = (size_t)XN * YN * Zi;
  const size_t plan = ddfan_plan_estimate_bytes(XN, YN, DNU, (int)Zi, (int)PNmax, sat_mode);
  if (!plan) return 0;
  size_t own = P * sizeof(ViewGeom) + P * (U + 1) * sizeof(double2) + P * U * sizeof(float) +
               3 * P * sizeof(int) + 2 * (size_t)numOfOS * sizeof(int) + P * U * sizeof(float) +
               (size_t)numOfOS * XN * YN * sizeof(float) + P * U * Zi * sizeof(float) +
               2 * V * sizeof(float) + PNmax * (U + (direct ? 1 : 0)) * Zi * sizeof(float) + sizeof(double);
  // direct mode: the initial image and the published copy (masked solves;
  // padded slices), sinogram staging and slice maps (padded slices)
  if (direct) {
    own += 2 * (size_t)XN * YN * SLN * sizeof(float);
    if (Zi != (size_t)SLN) own += P * U * SLN * sizeof(float) + (Zi + SLN) * sizeof(int);
  }
  sat_mode = cell_mode(sat_mode);  // the set-up's weight kernels keep tables
  // transient at creation: the one-slice weight plan and the slice-major
  // weight buffers (geometry, row sums, ones, tables) over nsub x PNmax rows
  const size_t R = (size_t)numOfOS * PNmax, CB = sat_mode == SAT_FP32 ? 8 : 16;
  const size_t weights = ddfan_plan_estimate_bytes(XN, YN, DNU, 1, 1, sat_mode) +
                         R * (sizeof(ViewGeom) + (U + 1) * sizeof(double2) + sizeof(float) + 3 * U * sizeof(float) +
                              (U + 1) * CB) +
                         (size_t)XN * YN * sizeof(float) + ((size_t)(XN + 2) * YN + (size_t)(YN + 2) * XN) * CB;
  return plan + own + weights;
}

DDFAN_API size_t ddfan_ossart_device_bytes(const ddfan_ossart* s) {
  return s ? reinterpret_cast<const Solver*>(s)->bytes : 0;
}

DDFAN_API int ddfan_ossart_set_sinogram(ddfan_ossart* h, const float* proj, int is_device, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || !proj) return set_err(DDFAN_ERR_ARG, "null argument");
  DeviceGuard g(s->device);
  const size_t n = (size_t)s->PNall * s->U * s->Z;
  cudaStream_t st = (cudaStream_t)stream;
  if (s->ps) {
    // slice-major [Z][PNall][U]
    const float* src = proj;
    if (!is_device) {
      DDFAN_CK(cudaMemcpyAsync(s->d_stage, proj, sizeof(float) * n, cudaMemcpyHostToDevice, st));
      src = s->d_stage;
    }
    int rc = ps_transpose(src, s->d_y, 1, (long long)s->PNall * s->U, s->Z, st);
    if (rc) return rc;
  } else if (!remapped(*s)) {
    DDFAN_CK(cudaMemcpyAsync(s->d_y, proj, sizeof(float) * n,
                             is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  } else {
    // into the internal slice order
    const float* src = proj;
    if (!is_device) {
      DDFAN_CK(cudaMemcpyAsync(s->d_stage, proj, sizeof(float) * n, cudaMemcpyHostToDevice, st));
      src = s->d_stage;
    }
    int rc = gather_slices(src, s->Z, s->d_y, s->Zi, s->d_perm, (size_t)s->PNall * s->U, st);
    if (rc) return rc;
  }
  cudaEventRecord(s->last_use, st);
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_set_image(ddfan_ossart* h, const float* img, int is_device, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || !img) return set_err(DDFAN_ERR_ARG, "null argument");
  DeviceGuard g(s->device);
  const size_t n = (size_t)s->XN * s->YN * s->Z;
  cudaStream_t st = (cudaStream_t)stream;
  if (s->ps) {
    DDFAN_CK(cudaMemcpyAsync(s->d_xu, img, sizeof(float) * n,
                             is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    int rc = ps_transpose(s->d_xu, s->d_x, 1, (long long)s->XN * s->YN, s->Z, st);
    if (rc) return rc;
  } else if (s->direct && (s->P->has_mask || s->Zi != s->Z)) {
    // masked and padded copy; the initial image kept where the mask is 0
    float* src = s->P->has_mask ? s->d_x0 : s->d_xu;
    DDFAN_CK(cudaMemcpyAsync(src, img, sizeof(float) * n,
                             is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    int rc = launch_stage_image(src, s->Z, s->P->has_mask ? s->P->d_mask : nullptr, s->d_x, s->Zi,
                                (size_t)s->XN * s->YN, st);
    if (rc) return rc;
  } else if (!s->win) {
    DDFAN_CK(cudaMemcpyAsync(s->d_x, img, sizeof(float) * n,
                             is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  } else {
    DDFAN_CK(cudaMemcpyAsync(s->d_xu, img, sizeof(float) * n,
                             is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    int rc = gather_slices(s->d_xu, s->Z, s->d_x, s->Zi, s->d_perm, (size_t)s->XN * s->YN, st);
    if (rc) return rc;
  }
  DDFAN_CK(cudaMemcpyAsync(s->d_xprev, s->d_x, sizeof(float) * (size_t)s->XN * s->YN * s->Zi,
                           cudaMemcpyDeviceToDevice, st));
  static const double one = 1.0;
  DDFAN_CK(cudaMemcpyAsync(s->d_t, &one, sizeof(double), cudaMemcpyHostToDevice, st));
  s->iters_done = 0;
  // the image callers read is the initial one until an iteration runs
  if (s->direct && published_copy(*s)) {
    int rc = solver_publish(*s, st);
    if (rc) return rc;
  }
  // the pageable host sources above must be consumed before returning
  DDFAN_CK(cudaStreamSynchronize(st));
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_iterate(ddfan_ossart* h, int numOfIter, int use_graph, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || numOfIter < 0) return set_err(DDFAN_ERR_ARG, "bad argument");
  DeviceGuard g(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (!use_graph) {
    for (int it = 0; it < numOfIter; ++it) {
      int rc = solver_iteration(*s, st);
      if (rc) return rc;
      ++s->iters_done;
    }
    int rc = solver_publish(*s, st);
    if (rc) return rc;
    cudaEventRecord(s->last_use, st);
    return DDFAN_OK;
  }
  if (!s->gexec) {
    DDFAN_CK(cudaStreamBeginCapture(s->own, cudaStreamCaptureModeThreadLocal));
    int rc = solver_iteration(*s, s->own);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->own, &gr);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    s->graph = gr;
    DDFAN_CK(cudaGraphInstantiate(&s->gexec, s->graph, 0));
  }
  for (int it = 0; it < numOfIter; ++it) {
    DDFAN_CK(cudaGraphLaunch(s->gexec, st));
    ++s->iters_done;
  }
  int rc = solver_publish(*s, st);
  if (rc) return rc;
  cudaEventRecord(s->last_use, st);
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_get_image(ddfan_ossart* h, float* img, int is_device, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || !img) return set_err(DDFAN_ERR_ARG, "null argument");
  DeviceGuard g(s->device);
  const size_t n = (size_t)s->XN * s->YN * s->Z;
  cudaStream_t st = (cudaStream_t)stream;
  DDFAN_CK(cudaMemcpyAsync(img, published_copy(*s) ? s->d_xu : s->d_x, sizeof(float) * n,
                           is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  cudaEventRecord(s->last_use, st);
  if (!is_device) DDFAN_CK(cudaStreamSynchronize(st));
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_profile(ddfan_ossart* h, int numOfIter, void* stream, float* ms_by_kind,
                                   int* launches_by_kind) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || numOfIter < 1 || !ms_by_kind || !launches_by_kind) return set_err(DDFAN_ERR_ARG, "bad argument");
  DeviceGuard g(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  LaunchProfiler prof;
  active_profiler() = &prof;
  int rc = DDFAN_OK;
  for (int it = 0; it < numOfIter && !rc; ++it) {
    rc = solver_iteration(*s, st);
    if (!rc) ++s->iters_done;
  }
  active_profiler() = nullptr;
  if (!rc) rc = solver_publish(*s, st);
  if (rc) return rc;
  DDFAN_CK(cudaStreamSynchronize(st));
  for (int k = 0; k < KIND_COUNT; ++k) {
    ms_by_kind[k] = 0.f;
    launches_by_kind[k] = 0;
  }
  for (size_t i = 0; i < prof.kind.size(); ++i) {
    float ms = 0.f;
    DDFAN_CK(cudaEventElapsedTime(&ms, prof.ev[2 * i], prof.ev[2 * i + 1]));
    ms_by_kind[prof.kind[i]] += ms;
    launches_by_kind[prof.kind[i]] += prof.kind[i] == KIND_FISTA ? 2 : 1;
  }
  return DDFAN_OK;
}

DDFAN_API float* ddfan_ossart_image_ptr(ddfan_ossart* h) {
  Solver* s = reinterpret_cast<Solver*>(h);
  return s ? (published_copy(*s) ? s->d_xu : s->d_x) : nullptr;
}

DDFAN_API int ddfan_ossart_launches_per_iter(const ddfan_ossart* h) {
  const Solver* s = reinterpret_cast<const Solver*>(h);
  if (!s) return 0;
  const bool adj = s->back_mode == DDFAN_BACK_ADJ;
  const int per = s->ps ? 7 : (s->direct ? (adj ? 3 : 2) : (adj ? 5 : 4));
  return s->nsub * per + (s->useFISTA ? 2 : 0);
}

DDFAN_API int ddfan_OSSART_AAPM(float x0, float y0, int DNU, const float* xds, const float* yds,
                                float detCntIdx, float imgXCenter, float imgYCenter, const float* proj,
                                const float* hangs, int PNall, int XN, int YN, int SLN, float dx,
                                const float* initImg, const uint8_t* mask, int numOfIter, int numOfOS,
                                int useFISTA, int nonneg, int sat_mode, int back_mode, float* reconImg) {
  if (!proj || !initImg || !reconImg) return set_err(DDFAN_ERR_ARG, "null argument");
  int dev = 0;
  cudaGetDevice(&dev);
  Solver* s = nullptr;
  int rc = solver_create(&s, x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, hangs, PNall, XN,
                         YN, SLN, dx, mask, numOfOS, useFISTA, nonneg, sat_mode, back_mode, dev);
  if (rc) return rc;
  ddfan_ossart* h = reinterpret_cast<ddfan_ossart*>(s);
  if (!rc) rc = ddfan_ossart_set_sinogram(h, proj, 0, s->own);
  if (!rc) rc = ddfan_ossart_set_image(h, initImg, 0, s->own);
  if (!rc) rc = ddfan_ossart_iterate(h, numOfIter, 1, s->own);
  if (!rc) rc = ddfan_ossart_get_image(h, reconImg, 0, s->own);
  solver_free(s);
  return rc;
}

}  // extern "C"
