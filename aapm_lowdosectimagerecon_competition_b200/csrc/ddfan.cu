// ddfan.cu -- host side of libddfan: plans, launches, the C ABI (include/ddfan.h).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_kernels.cuh"
#include "ddfan_plan.h"
#include "ddfan_ps.h"

namespace ddfan {

// ------------------------------------------------------------------ errors

static thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

const char* last_error() { return g_err.c_str(); }

// ------------------------------------------------------------------ profiler

LaunchProfiler*& active_profiler() {
  static thread_local LaunchProfiler* p = nullptr;
  return p;
}

int LaunchProfiler::mark(int k, cudaStream_t st) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    cudaGetLastError();
    return -1;
  }
  cudaEventRecord(a, st);
  ev.push_back(a);
  ev.push_back(b);
  kind.push_back(k);
  return (int)kind.size() - 1;
}

void LaunchProfiler::done(int slot, cudaStream_t st) { cudaEventRecord(ev[2 * slot + 1], st); }

LaunchProfiler::~LaunchProfiler() {
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
}

// ------------------------------------------------------------------ plan

// Tile widths chosen by the autotuner (ddfan_tune_set_zl), keyed by the
// number of 4-slice blocks; consulted before the built-in cost model.
static std::mutex g_tune_mutex;
static std::map<int, int> g_tuned_zl;
static std::map<int, int> g_tuned_nz;  // z-tiles per thread of the direct kernels

static int tuned_zl(int ZB) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tuned_zl.find(ZB);
  return it == g_tuned_zl.end() ? 0 : it->second;
}

// z-blocks per z-tile: wider tiles gather more contiguous bytes per request,
// but a stack of ZB blocks is padded to whole tiles.  Relative cost per
// padded block of each width (measured on the 512^2 x 128 workload: widths
// 8, 4, 2 ran at 1 : 1.2 : 2.1); pick the cheapest padded stack, unless the
// autotuner recorded a measured choice for this stack.
int pow2_zl(int ZB) {
  const int t = tuned_zl(ZB);
  if (t == 1 || t == 2 || t == 4 || t == 8)
    if (t <= ZB) return t;
  const int widths[4] = {8, 4, 2, 1};
  const double cost[4] = {1.0, 1.2, 2.1, 3.6};
  int best = 1;
  double bc = 1e300;
  for (int i = 0; i < 4; ++i) {
    const int w = widths[i];
    if (w > ZB) continue;
    const double c = (double)((ZB + w - 1) / w * w) * cost[i];
    if (c < bc) { bc = c; best = w; }
  }
  return best;
}

int plan_nz(int ZB) {
  if (const char* v = getenv("DDFAN_NZ")) {  // a fixed value for measurements, like DDFAN_ZL
    const int nz = atoi(v);
    if (nz == 1 || nz == 2 || nz == 4) return nz;
  }
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tuned_nz.find(ZB);
  return it == g_tuned_nz.end() ? DDFAN_DD_NZ : it->second;
}

int plan_zl(int ZB, int zl_force) {
  int ZL = pow2_zl(ZB);
  if (const char* zl = getenv("DDFAN_ZL")) {
    const int v = atoi(zl);
    if ((v == 1 || v == 2 || v == 4 || v == 8) && v <= ZL) ZL = v;
  }
  if (zl_force == 1 || zl_force == 2 || zl_force == 4 || zl_force == 8) ZL = zl_force;
  return ZL;
}

// Stream-ordered device memory from one pool per device owned by the
// library: creating or destroying a plan or a solver never synchronises the
// device, so other solves keep running meanwhile.  The pool keeps the blocks
// that destroyed plans and solvers free (release threshold: unlimited) and
// serves the next ones from them; the device's default pool returns freed
// memory to the driver at every synchronisation, and mapping it again cost
// 30 ms to 1 s per gigabyte-sized solve.  ddfan_release_cached hands the
// unused part back.
static std::mutex g_pool_mutex;
static std::map<int, cudaMemPool_t> g_pools;

static cudaMemPool_t lib_pool(int dev, bool create) {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) return it->second;
  if (!create) return nullptr;
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pools[dev] = pool;
  return pool;
}

int dev_alloc(void** p, size_t bytes, cudaStream_t st) {
  *p = nullptr;
  bytes = std::max<size_t>(bytes, 1);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool = lib_pool(dev, true);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
  if (e == cudaErrorMemoryAllocation && pool) {
    // cached blocks too fragmented for this request: give them back, retry once
    cudaGetLastError();
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(DDFAN_ERR_NOMEM, "cudaMallocFromPoolAsync(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  return DDFAN_OK;
}

void dev_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

template <class T>
static int dalloc(T** p, size_t n, size_t* bytes, cudaStream_t st) {
  if (n == 0) n = 1;
  int rc = dev_alloc((void**)p, n * sizeof(T), st);
  if (!rc) *bytes += n * sizeof(T);
  return rc;
}

// Releases a plan's device memory once the plan's last recorded use
// (mark_use) has completed; does not block the host.
void plan_free(Plan* P) {
  if (!P) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(P->device);
  if (P->alloc_stream) {
    if (P->last_use) cudaStreamWaitEvent(P->alloc_stream, P->last_use, 0);
    void* ptrs[] = {P->d_bx, P->d_by, P->d_xd, P->d_yd, P->d_mask, P->d_tb, P->d_lut, P->d_satx,
                    P->d_saty, P->d_satq, P->d_vg, P->d_fc, P->d_cvd, P->d_tmp, P->d_angs,
                    P->d_order, P->d_counts, P->ps_ang, P->ps_vg, P->ps_fc, P->ps_cvd, P->ps_img,
                    P->ps_imgt, P->ps_sino, P->ps_tabx, P->ps_taby, P->ps_sq};
    for (void* q : ptrs) dev_free(q, P->alloc_stream);
    cudaStreamDestroy(P->alloc_stream);
  }
  if (P->last_use) cudaEventDestroy(P->last_use);
  cudaGetLastError();
  if (prev >= 0) cudaSetDevice(prev);
  delete P;
}

void mark_use(Plan& p, cudaStream_t st) {
  if (p.last_use) cudaEventRecord(p.last_use, st);
}

// DD3Boundaries (AAPM_script/utilities.cuh:268-287): evaluated in double,
// stored as float like the reference's float arrays.
void boundaries(int n, const float* c, std::vector<double>& out) {
  const int nb = n + 1;
  out.assign(nb, 0.0);
  if (nb >= 3) {
    for (int i = 0; i < nb; ++i) {
      double v;
      if (i == 0) v = 1.5 * c[0] - 0.5 * c[1];
      else if (i == nb - 1) v = 1.5 * c[i - 1] - 0.5 * c[i - 2];
      else v = 0.5 * c[i - 1] + 0.5 * c[i];
      out[i] = (double)(float)v;
    }
  } else {
    out[0] = (double)(float)(c[0] - 0.5);
    out[1] = (double)(float)(c[0] + 0.5);
  }
}

// The direct forward kernels' dynamic shared memory, allowed on the current
// device (dev, for the message) at every plan creation -- a kernel
// attribute belongs to the context, which a device reset replaces.  Plan
// creation precedes every launch on a plan and never runs under capture.
int dd_prepare_device(int dev) {
  cudaError_t e = cudaSuccess;
#define DDFAN_DD_ALLOW(ZLv, NZv)                                                                  \
  if (e == cudaSuccess)                                                                           \
    e = dd_allow_dyn(k_fwd_dd<ZLv, DdFwdCG<ZLv>::v, NZv>, DdFwdTile<ZLv, DdFwdCG<ZLv>::v, NZv>::DYN);
  DDFAN_DD_ALLOW(8, 4) DDFAN_DD_ALLOW(8, 2) DDFAN_DD_ALLOW(8, 1)
  DDFAN_DD_ALLOW(4, 4) DDFAN_DD_ALLOW(4, 2) DDFAN_DD_ALLOW(4, 1)
  DDFAN_DD_ALLOW(2, 4) DDFAN_DD_ALLOW(2, 2) DDFAN_DD_ALLOW(2, 1)
  DDFAN_DD_ALLOW(1, 4) DDFAN_DD_ALLOW(1, 2) DDFAN_DD_ALLOW(1, 1)
#undef DDFAN_DD_ALLOW
  if (e != cudaSuccess)
    return set_err(DDFAN_ERR_CUDA, "forward kernel attributes on device %d: %s", dev, cudaGetErrorString(e));
  return DDFAN_OK;
}

int plan_create(Plan** out, const PlanDesc& d) {
  *out = nullptr;
  if (d.DNU < 2 || d.XN < 1 || d.YN < 1 || d.SLN < 1 || d.PNmax < 1 || !d.xds || !d.yds)
    return set_err(DDFAN_ERR_ARG, "plan: bad sizes (DNU=%d XN=%d YN=%d SLN=%d PNmax=%d) or null geometry",
                   d.DNU, d.XN, d.YN, d.SLN, d.PNmax);
  if (!(d.dx > 0.f)) return set_err(DDFAN_ERR_ARG, "plan: dx must be > 0");
  if (d.sat_mode < SAT_FP32 || d.sat_mode > SAT_DIRECT) return set_err(DDFAN_ERR_ARG, "plan: sat_mode %d", d.sat_mode);
  if (d.XN > 1024 || d.YN > 1024 || d.DNU + 1 > 1024)
    return set_err(DDFAN_ERR_UNSUPPORTED, "plan: lines longer than 1024 cells are not supported");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "no CUDA device");
  }
  if (d.device < 0 || d.device >= ndev) return set_err(DDFAN_ERR_ARG, "device %d of %d", d.device, ndev);
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(d.device) != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "cudaSetDevice(%d)", d.device);
  {
    const int rc = dd_prepare_device(d.device);
    if (rc) {
      if (prev >= 0) cudaSetDevice(prev);
      return rc;
    }
  }
  std::unique_ptr<Plan, void (*)(Plan*)> P(new Plan(), plan_free);
  Plan& p = *P;
  p.device = d.device;
  p.XN = d.XN; p.YN = d.YN; p.U = d.DNU; p.Z = d.SLN; p.ZB = (d.SLN + 3) / 4;
  p.PNmax = d.PNmax; p.mode = d.sat_mode; p.ZL = plan_zl(p.ZB, d.zl_force); p.NZ = plan_nz(p.ZB);
  p.P4 = p.ZB;
  // whole z-tiles: the padding blocks of the last tile are never written; the
  // projectors read them only for the slices past Z, whose results they drop
  p.ZB = (p.ZB + p.ZL - 1) / p.ZL * p.ZL;
  p.x0 = d.x0; p.y0 = d.y0; p.dx = d.dx; p.detCntIdx = d.detCntIdx;
  p.ocx = (d.XN - 1.0) * 0.5 - (double)d.imgXCenter / (double)d.dx;
  p.ocy = (d.YN - 1.0) * 0.5 - (double)d.imgYCenter / (double)d.dx;
  boundaries(d.DNU, d.xds, p.bx);
  boundaries(d.DNU, d.yds, p.by);
  p.xd.assign(d.xds, d.xds + d.DNU);
  p.yd.assign(d.yds, d.yds + d.DNU);
  // REF backprojector constants (AAPM_script/MultiSlicesBackGPU.cu:141, :150, :211, :226-227)
  {
    const double S2D = std::hypot((double)d.xds[0] - d.x0, (double)d.yds[0] - d.y0);
    const double ex = (double)d.xds[1] - d.xds[0], ey = (double)d.yds[1] - d.yds[0];
    const double dbeta = std::atan(std::sqrt(ex * ex + ey * ey) / S2D * 0.5) * 2.0;
    p.inv_dbeta = 1.0 / dbeta;
    p.inv_sid = 1.0 / std::sqrt((double)d.x0 * d.x0 + (double)d.y0 * d.y0);
  }
  // exact-adjoint bracket table: fan tangent of every boundary, seen from the source
  {
    const double sl = std::sqrt((double)d.x0 * d.x0 + (double)d.y0 * d.y0);
    if (!(sl > 0)) return set_err(DDFAN_ERR_ARG, "source at the rotation centre");
    p.sh0x = -d.x0 / sl; p.sh0y = -d.y0 / sl;
    std::vector<double> T(d.DNU + 1);
    for (int b = 0; b <= d.DNU; ++b) {
      const double vx = p.bx[b] - d.x0, vy = p.by[b] - d.y0;
      T[b] = (p.sh0x * vy - p.sh0y * vx) / (p.sh0x * vx + p.sh0y * vy);
    }
    p.dirt = T[d.DNU] >= T[0] ? 1.f : -1.f;
    p.tb.resize(d.DNU + 1);
    bool mono = true;
    for (int b = 0; b <= d.DNU; ++b) {
      p.tb[b] = (float)(p.dirt * T[b]);
      if (b && !(p.tb[b] > p.tb[b - 1])) mono = false;
    }
    p.adj_ok = mono;
    p.M = 4 * (d.DNU + 1);
    p.t0 = p.tb[0];
    const double span = (double)p.tb[d.DNU] - p.tb[0];
    p.invdt = (float)(p.M / span);
    p.lut.resize(p.M);
    int b = 0;
    for (int m = 0; m < p.M; ++m) {
      const double tm = p.tb[0] + m * span / p.M;
      while (b < d.DNU && p.tb[b + 1] <= tm) ++b;
      p.lut[m] = (uint16_t)std::min(b, d.DNU - 1);
    }
  }
  size_t& B = p.bytes;
  int rc;
  if (cudaStreamCreateWithFlags(&p.alloc_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p.last_use, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    return set_err(DDFAN_ERR_CUDA, "plan: stream/event creation failed");
  }
  cudaStream_t as = p.alloc_stream;
  const bool direct = p.mode == SAT_DIRECT;
  const size_t F4 = cell_f4(p.mode);
  // direct mode: no image tables; the staged sinogram operand [PNmax][U+1][P4]
  // float4 and a staged image of 4 P4 slices
  const size_t nimg = direct ? 0 : (size_t)p.XN * p.YN * p.ZB * F4;
  const size_t nsino = direct ? (size_t)p.PNmax * (p.U + 1) * p.P4 : (size_t)p.PNmax * (p.U + 1) * p.ZB * F4;
  const size_t ntmp = (size_t)p.XN * p.YN * (direct ? 4 * (size_t)p.P4 : (size_t)p.Z);
  if ((rc = dalloc(&p.d_bx, p.U + 1, &B, as)) || (rc = dalloc(&p.d_by, p.U + 1, &B, as)) ||
      (rc = dalloc(&p.d_xd, p.U, &B, as)) || (rc = dalloc(&p.d_yd, p.U, &B, as)) ||
      (rc = dalloc(&p.d_mask, (size_t)p.XN * p.YN, &B, as)) || (rc = dalloc(&p.d_tb, p.U + 1, &B, as)) ||
      (rc = dalloc(&p.d_lut, p.M, &B, as)) || (!direct && (rc = dalloc(&p.d_satx, nimg, &B, as))) ||
      (!direct && (rc = dalloc(&p.d_saty, nimg, &B, as))) || (rc = dalloc(&p.d_satq, nsino, &B, as)) ||
      (rc = dalloc(&p.d_vg, p.PNmax, &B, as)) || (rc = dalloc(&p.d_fc, (size_t)p.PNmax * (p.U + 1), &B, as)) ||
      (rc = dalloc(&p.d_cvd, (size_t)p.PNmax * p.U, &B, as)) ||
      (rc = dalloc(&p.d_tmp, ntmp, &B, as)) ||
      (rc = dalloc(&p.d_angs, (size_t)p.PNmax, &B, as)) ||
      (rc = dalloc(&p.d_order, (size_t)p.PNmax, &B, as)) || (rc = dalloc(&p.d_counts, 2, &B, as))) {
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
  }
  std::vector<uint8_t> m((size_t)p.XN * p.YN, 1);
  if (d.mask) std::memcpy(m.data(), d.mask, m.size());
  p.has_mask = d.mask != nullptr;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_bx, p.bx.data(), sizeof(double) * (p.U + 1), cudaMemcpyHostToDevice, as);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_by, p.by.data(), sizeof(double) * (p.U + 1), cudaMemcpyHostToDevice, as);
  std::vector<double> xd(p.xd.begin(), p.xd.end()), yd(p.yd.begin(), p.yd.end());
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_xd, xd.data(), sizeof(double) * p.U, cudaMemcpyHostToDevice, as);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_yd, yd.data(), sizeof(double) * p.U, cudaMemcpyHostToDevice, as);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_mask, m.data(), m.size(), cudaMemcpyHostToDevice, as);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_tb, p.tb.data(), sizeof(float) * (p.U + 1), cudaMemcpyHostToDevice, as);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_lut, p.lut.data(), sizeof(uint16_t) * p.M, cudaMemcpyHostToDevice, as);
  // the allocations and the staged uploads complete before the plan is used on any stream
  if (e == cudaSuccess) e = cudaStreamSynchronize(as);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "plan upload: %s", cudaGetErrorString(e));
  *out = P.release();
  return DDFAN_OK;
}

// ------------------------------------------------------------------ launches

static int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return DDFAN_OK;
}

static GeomConsts geom_consts(const Plan& p) {
  GeomConsts g;
  g.x0 = p.x0; g.y0 = p.y0; g.dx = p.dx; g.ocx = p.ocx; g.ocy = p.ocy;
  g.bx = p.d_bx; g.by = p.d_by; g.xd = p.d_xd; g.yd = p.d_yd;
  g.sh0x = p.sh0x; g.sh0y = p.sh0y;
  g.U = p.U; g.XN = p.XN; g.YN = p.YN;
  return g;
}

int launch_view_geom(const Plan& p, const float* d_angs, int stride, int PN, ViewGeom* vg,
                     double2* fc, float* cvd, cudaStream_t st) {
  if (PN < 1) return set_err(DDFAN_ERR_ARG, "PN must be >= 1");
  ProfScope ps(KIND_VIEW_GEOM, st);
  k_view_geom<<<PN, 128, 0, st>>>(geom_consts(p), d_angs, stride, PN, vg, fc, cvd);
  return check_launch("k_view_geom");
}

template <int M>
static int sat_dispatch(const SatSrc& s, float4* out0, int nl0, float4* out1, int nl1, int N0, int N1,
                        int Nw0, int Nw1, int ZB, int ntab, cudaStream_t st) {
  const int Nw = std::max(Nw0, Nw1);
  dim3 grid(std::max(nl0, nl1), (s.zb1 - s.zb0 + 7) / 8, ntab);
  // 512 threads = 8 z lanes x 64 chunks of C cells
  if (Nw <= 64 * 2) k_sat<M, 2><<<grid, 512, 0, st>>>(s, out0, nl0, nl1, out1, N0, N1, Nw0, Nw1, ZB);
  else if (Nw <= 64 * 4) k_sat<M, 4><<<grid, 512, 0, st>>>(s, out0, nl0, nl1, out1, N0, N1, Nw0, Nw1, ZB);
  else if (Nw <= 64 * 8) k_sat<M, 8><<<grid, 512, 0, st>>>(s, out0, nl0, nl1, out1, N0, N1, Nw0, Nw1, ZB);
  else if (Nw <= 64 * 12) k_sat<M, 12><<<grid, 512, 0, st>>>(s, out0, nl0, nl1, out1, N0, N1, Nw0, Nw1, ZB);
  else if (Nw <= 64 * 16) k_sat<M, 16><<<grid, 512, 0, st>>>(s, out0, nl0, nl1, out1, N0, N1, Nw0, Nw1, ZB);
  else return set_err(DDFAN_ERR_UNSUPPORTED, "line of %d cells", Nw);
  return check_launch("k_sat");
}

static int sat_launch(int mode, const SatSrc& s, float4* out0, int nl0, float4* out1, int nl1, int N0,
                      int N1, int Nw0, int Nw1, int ZB, int ntab, cudaStream_t st) {
  switch (mode) {
    case SAT_FP32: return sat_dispatch<SAT_FP32>(s, out0, nl0, out1, nl1, N0, N1, Nw0, Nw1, ZB, ntab, st);
    case SAT_HILO: return sat_dispatch<SAT_HILO>(s, out0, nl0, out1, nl1, N0, N1, Nw0, Nw1, ZB, ntab, st);
    case SAT_FP64: return sat_dispatch<SAT_FP64>(s, out0, nl0, out1, nl1, N0, N1, Nw0, Nw1, ZB, ntab, st);
  }
  return set_err(DDFAN_ERR_ARG, "sat mode %d", mode);
}

// Both image tables (rows -> satx, columns -> saty) in one launch; the mask
// multiply of AAPM_script/MultiSlicesProjGPU.cu:202-209 happens on load.
// z-blocks holding slices [zlo, zhi)
static void zblock_range(const Plan& p, int zlo, int zhi, int* zb0, int* zb1) {
  if (zhi < 0 || zhi > p.Z) zhi = p.Z;
  zlo = std::max(0, std::min(zlo, zhi));
  *zb0 = zlo / 4;
  *zb1 = std::max(*zb0, (zhi + 3) / 4);
}

// z-tiles (ZL z-blocks each) holding slices [zlo, zhi)
static void ztile_range(const Plan& p, int zlo, int zhi, int* zt0, int* nzt) {
  int zb0, zb1;
  zblock_range(p, zlo, zhi, &zb0, &zb1);
  *zt0 = zb0 / p.ZL;
  *nzt = zb1 > zb0 ? (zb1 + p.ZL - 1) / p.ZL - *zt0 : 0;
}

int launch_sat_image(const Plan& p, const float* d_vol, cudaStream_t st, int zlo, int zhi) {
  SatSrc s{};
  s.kind = 0; s.a = d_vol; s.mask = p.has_mask ? p.d_mask : nullptr;
  s.XN = p.XN; s.YN = p.YN; s.U = p.U; s.Z = p.Z; s.ZLt = p.ZL;
  zblock_range(p, zlo, zhi, &s.zb0, &s.zb1);
  if (s.zb1 <= s.zb0) return DDFAN_OK;
  ProfScope ps(KIND_SAT_IMAGE, st);
  return sat_launch(p.mode, s, p.d_satx, p.YN, p.d_saty, p.XN, p.XN, p.YN, p.XN, p.YN, p.ZB, 2, st);
}

int launch_sat_sino(const Plan& p, const float* d_prj, int PN, const float* wgt, float wscale,
                    const float* y, const int* yview, const float* rowsum, cudaStream_t st, int zlo,
                    int zhi, const ViewRanges* vr) {
  SatSrc s{};
  s.kind = 2; s.a = d_prj; s.wgt = wgt; s.wscale = wscale; s.y = y; s.yview = yview;
  s.rowsum = rowsum; s.XN = p.XN; s.YN = p.YN; s.U = p.U; s.Z = p.Z; s.ZLt = p.ZL;
  if (vr) {
    s.ztd = vr->ztd; s.soff = vr->soff; s.Mc = vr->Mc; s.nOS = vr->nOS; s.ksub = vr->ksub; s.T = vr->T;
  }
  zblock_range(p, zlo, zhi, &s.zb0, &s.zb1);
  if (s.zb1 <= s.zb0) return DDFAN_OK;
  ProfScope ps(KIND_SAT_SINO, st);
  return sat_launch(p.mode, s, p.d_satq, PN, nullptr, 0, p.U, 0, p.U + 1, 0, p.ZB, 1, st);
}

// Views of a call in dispatch order (x-major first) and their counts.
int launch_view_order(const ViewGeom* vg, int PN, int* order, int* counts, cudaStream_t st) {
  ProfScope ps(KIND_VIEW_GEOM, st);
  k_view_order<<<1, 1024, 0, st>>>(vg, PN, order, counts);
  return check_launch("k_view_order");
}

int launch_view_order_ranges(const ViewGeom* vg, int4* desc, int nr, int* order, cudaStream_t st) {
  if (nr < 1) return DDFAN_OK;
  ProfScope ps(KIND_VIEW_GEOM, st);
  k_view_order_ranges<<<nr, 1024, 0, st>>>(vg, desc, order);
  return check_launch("k_view_order_ranges");
}

// channels per thread of the forward projector for a z-lane count
template <int ZL> struct FwdCG { static constexpr int v = ZL >= 4 ? 4 : (ZL == 2 ? 2 : 1); };

template <int M, int ZL>
static void fwd_go(const FwdArgs& a, int nzt, cudaStream_t st) {
  constexpr int CG = FwdCG<ZL>::v;
  using T = FwdTile<ZL, CG>;
  constexpr int kMaxRows = 65535;  // grid y limit
  for (int r0 = 0; r0 < a.PN; r0 += kMaxRows) {
    FwdArgs b = a;
    b.row0 = r0;
    dim3 grid((a.U + T::CW - 1) / T::CW, std::min(a.PN - r0, kMaxRows), nzt);
    k_fwd<M, ZL, CG><<<grid, T::NT, 0, st>>>(b);
  }
}

template <int M>
static void fwd_zl(int ZL, const FwdArgs& a, int nzt, cudaStream_t st) {
  switch (ZL) {
    case 8: fwd_go<M, 8>(a, nzt, st); break;
    case 4: fwd_go<M, 4>(a, nzt, st); break;
    case 2: fwd_go<M, 2>(a, nzt, st); break;
    default: fwd_go<M, 1>(a, nzt, st); break;
  }
}

int launch_fwd(const Plan& p, const ViewGeom* vg, const double2* fc, const float* cvd,
               const int* order, int PN, float* d_prj, int zlo, int zhi, cudaStream_t st,
               const int4* ztd) {
  FwdArgs a;
  a.row0 = 0;
  a.ztd = ztd;
  a.satx = p.d_satx; a.saty = p.d_saty; a.vg = vg; a.fc = fc; a.cvd = cvd; a.order = order;
  a.out = d_prj; a.PN = PN; a.U = p.U; a.Z = p.Z; a.ZB = p.ZB; a.XN = p.XN; a.YN = p.YN;
  a.dx = p.dx; a.zlo = zlo; a.zhi = zhi;
  int nzt = 0;
  ztile_range(p, zlo, zhi, &a.zt0, &nzt);
  if (nzt == 0) return DDFAN_OK;
  ProfScope ps(KIND_FWD, st);
  switch (p.mode) {
    case SAT_FP32: fwd_zl<SAT_FP32>(p.ZL, a, nzt, st); break;
    case SAT_HILO: fwd_zl<SAT_HILO>(p.ZL, a, nzt, st); break;
    default: fwd_zl<SAT_FP64>(p.ZL, a, nzt, st); break;
  }
  return check_launch("k_fwd");
}

template <int M, int ZL>
static void ref_go(const RefArgs& a, int nzt, cudaStream_t st) {
  using T = BackTile<ZL>;
  const int tiles = ((a.YN + T::LT - 1) / T::LT) * ((a.XN + T::KT - 1) / T::KT);
  dim3 grid(tiles, 1, nzt);
  k_back_ref<M, ZL><<<grid, T::NT, 0, st>>>(a);
}

template <int M, int ZL, bool XM>
static void adj_go(const AdjArgs& a, int nzt, cudaStream_t st) {
  using T = BackTile<ZL>;
  const int nl = XM ? a.XN : a.YN, N = XM ? a.YN : a.XN;
  const int tiles = ((nl + T::LT - 1) / T::LT) * ((N + T::KT - 1) / T::KT);
  dim3 grid(tiles, 1, nzt);
  k_back_adj<M, ZL, XM><<<grid, T::NT, 0, st>>>(a);
}

template <int M>
static void ref_zl(int ZL, const RefArgs& a, int nzt, cudaStream_t st) {
  switch (ZL) {
    case 8: ref_go<M, 8>(a, nzt, st); break;
    case 4: ref_go<M, 4>(a, nzt, st); break;
    case 2: ref_go<M, 2>(a, nzt, st); break;
    default: ref_go<M, 1>(a, nzt, st); break;
  }
}

template <int M, bool XM>
static void adj_zl(int ZL, const AdjArgs& a, int nzt, cudaStream_t st) {
  switch (ZL) {
    case 8: adj_go<M, 8, XM>(a, nzt, st); break;
    case 4: adj_go<M, 4, XM>(a, nzt, st); break;
    case 2: adj_go<M, 2, XM>(a, nzt, st); break;
    default: adj_go<M, 1, XM>(a, nzt, st); break;
  }
}

// Backprojection of the table in p.d_satq (built by launch_sat_sino with the
// matching weights).  `epi` holds the final destination/update; ADJ runs two
// passes (x-column lines over the x-major views, then y-row lines over the
// others) through p.d_tmp.  order/counts come from launch_view_order.
int launch_back(const Plan& p, int back_mode, const ViewGeom* vg, const double2* fc,
                const int* order, const int* counts, int PN, const BackEpi& epi, cudaStream_t st,
                const int4* ztd) {
  int zt0 = 0, nzt = 0;
  ztile_range(p, epi.zlo, epi.zhi, &zt0, &nzt);
  if (nzt == 0) return DDFAN_OK;
  if (back_mode == DDFAN_BACK_REF) {
    RefArgs a;
    a.satq = p.d_satq; a.vg = vg; a.PN = PN; a.U = p.U; a.Z = p.Z; a.ZB = p.ZB;
    a.XN = p.XN; a.YN = p.YN; a.ocx = p.ocx; a.ocy = p.ocy; a.dx = p.dx;
    a.inv_sid = p.inv_sid; a.inv_dbeta = p.inv_dbeta; a.cnt = (double)p.detCntIdx + 0.5;
    a.epi = epi;
    a.zt0 = zt0;
    a.ztd = ztd;
    ProfScope ps(KIND_BACK_A, st);
    switch (p.mode) {
      case SAT_FP32: ref_zl<SAT_FP32>(p.ZL, a, nzt, st); break;
      case SAT_HILO: ref_zl<SAT_HILO>(p.ZL, a, nzt, st); break;
      default: ref_zl<SAT_FP64>(p.ZL, a, nzt, st); break;
    }
    return check_launch("k_back_ref");
  }
  if (back_mode != DDFAN_BACK_ADJ) return set_err(DDFAN_ERR_ARG, "back_mode %d", back_mode);
  if (!p.adj_ok) return set_err(DDFAN_ERR_UNSUPPORTED, "detector boundaries are not monotone as seen from the source");
  if (!order || (!counts && !ztd)) return set_err(DDFAN_ERR_ARG, "exact adjoint needs the view order");
  AdjArgs a;
  a.ztd = ztd;
  a.satq = p.d_satq; a.vg = vg; a.fc = fc; a.tb = p.d_tb; a.lut = p.d_lut;
  a.order = order; a.counts = counts;
  a.t0 = p.t0; a.invdt = p.invdt; a.dirt = p.dirt; a.M = p.M;
  a.PN = PN; a.U = p.U; a.Z = p.Z; a.ZB = p.ZB; a.XN = p.XN; a.YN = p.YN;
  a.ocx = p.ocx; a.ocy = p.ocy; a.dx = p.dx;
  a.zt0 = zt0;
  // pass 1: x-major views, lines = x columns -> tmp (mask applied)
  a.epi = epi;
  a.epi.out = p.d_tmp; a.epi.addend = nullptr; a.epi.xin = nullptr; a.epi.colsum = nullptr;
  a.epi.nonneg = 0;
  {
    ProfScope ps(KIND_BACK_A, st);
    switch (p.mode) {
      case SAT_FP32: adj_zl<SAT_FP32, true>(p.ZL, a, nzt, st); break;
      case SAT_HILO: adj_zl<SAT_HILO, true>(p.ZL, a, nzt, st); break;
      default: adj_zl<SAT_FP64, true>(p.ZL, a, nzt, st); break;
    }
  }
  int rc = check_launch("k_back_adj<x>");
  if (rc) return rc;
  // pass 2: y-major views, lines = y rows, plus pass 1, then the final epilogue
  a.epi = epi;
  a.epi.addend = p.d_tmp;
  {
    ProfScope ps(KIND_BACK_B, st);
    switch (p.mode) {
      case SAT_FP32: adj_zl<SAT_FP32, false>(p.ZL, a, nzt, st); break;
      case SAT_HILO: adj_zl<SAT_HILO, false>(p.ZL, a, nzt, st); break;
      default: adj_zl<SAT_FP64, false>(p.ZL, a, nzt, st); break;
    }
  }
  return check_launch("k_back_adj<y>");
}

// ------------------------------------------------------------------ direct mode

static int grid_blocks(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

int launch_stage_image(const float* src, int Z, const uint8_t* mask, float* dst, int Zp, size_t npix,
                       cudaStream_t st) {
  k_stage_image<<<grid_blocks(npix * Zp), 256, 0, st>>>(src, Z, mask, dst, Zp, npix);
  return check_launch("k_stage_image");
}

int launch_stage_sino(const float* src, int Z, const float* wgt, int U, float* dst, int Zp, size_t PN,
                      cudaStream_t st) {
  ProfScope ps(KIND_SAT_SINO, st);
  k_stage_sino<<<grid_blocks(PN * (U + 1) * Zp), 256, 0, st>>>(src, Z, wgt, U, dst, Zp, PN);
  return check_launch("k_stage_sino");
}

int launch_publish_masked(const float* x, int Zi, const float* x0, int Z, const uint8_t* mask, int clamp0,
                          float* out, size_t npix, cudaStream_t st) {
  k_publish_masked<<<grid_blocks(npix * Z), 256, 0, st>>>(x, Zi, x0, Z, mask, clamp0, out, npix);
  return check_launch("k_publish_masked");
}

template <int ZL>
static void fwd_dd_go(const DdFwdArgs& a, int nzt, cudaStream_t st) {
  constexpr int CG = DdFwdCG<ZL>::v;
  constexpr int kMaxRows = DDFAN_DD_FWD_ROWS_X ? (1 << 30) : 65535;  // grid x / y limit
  const auto go = [&](auto nz) {
    constexpr int NZ = decltype(nz)::value;
    using T = DdFwdTile<ZL, CG, NZ>;
    for (int r0 = 0; r0 < a.PN; r0 += kMaxRows) {
      DdFwdArgs b = a;
      b.row0 = r0;
      const int rows = std::min(a.PN - r0, kMaxRows), cblk = (a.U + T::CW - 1) / T::CW;
      const dim3 grid(DDFAN_DD_FWD_ROWS_X ? rows : cblk, DDFAN_DD_FWD_ROWS_X ? cblk : rows, (nzt + NZ - 1) / NZ);
      k_fwd_dd<ZL, CG, NZ><<<grid, T::NT, T::DYN, st>>>(b);
    }
  };
  switch (dd_nz(nzt, a.nzc)) {
    case 4: go(std::integral_constant<int, 4>()); break;
    case 2: go(std::integral_constant<int, 2>()); break;
    default: go(std::integral_constant<int, 1>()); break;
  }
}

DdFwdArgs make_fwd_dd_args(const Plan& p, const float* img, const ViewGeom* vg, const double2* fc,
                           const float* cvd, const int* order, int PN, float* out, int orow, int ostride, int zlo,
                           int zhi, const DdResidual* res) {
  DdFwdArgs a{};
  a.img = reinterpret_cast<const float4*>(img); a.P4 = p.P4;
  a.vg = vg; a.fc = fc; a.cvd = cvd; a.order = order;
  a.out = out; a.orow = orow; a.ostride = ostride;
  a.PN = PN; a.U = p.U; a.Z = p.Z; a.XN = p.XN; a.YN = p.YN; a.dx = (float)p.dx;
  a.zlo = zlo; a.zhi = zhi < 0 ? p.Z : zhi; a.row0 = 0; a.nzc = p.NZ;
  if (res) {
    a.y = res->y; a.yview = res->yview; a.rowsum = res->rowsum; a.wgt = res->wgt; a.ystride = res->ystride;
  }
  ztile_range(p, zlo, zhi, &a.zt0, &a.nzt);
  return a;
}

int launch_fwd_dd(const Plan& p, const float* img, const ViewGeom* vg, const double2* fc, const float* cvd,
                  const int* order, int PN, float* out, int orow, int ostride, int zlo, int zhi,
                  const DdResidual* res, cudaStream_t st) {
  const DdFwdArgs a = make_fwd_dd_args(p, img, vg, fc, cvd, order, PN, out, orow, ostride, zlo, zhi, res);
  const int nzt = a.nzt;
  if (nzt == 0 || PN < 1) return DDFAN_OK;
  ProfScope ps(KIND_FWD, st);
  switch (p.ZL) {
    case 8: fwd_dd_go<8>(a, nzt, st); break;
    case 4: fwd_dd_go<4>(a, nzt, st); break;
    case 2: fwd_dd_go<2>(a, nzt, st); break;
    default: fwd_dd_go<1>(a, nzt, st); break;
  }
  return check_launch("k_fwd_dd");
}

template <int ZL, bool XM>
static void back_dd_go(const DdAdjArgs& a, int nzt, cudaStream_t st) {
  using T = DdBackTile<ZL>;
  const int nl = XM ? a.XN : a.YN, N = XM ? a.YN : a.XN;
  const int tiles = ((nl + T::LT - 1) / T::LT) * ((N + T::KT - 1) / T::KT);
  switch (dd_nz(nzt, a.nzc)) {
    case 4: k_back_dd<ZL, XM, 4><<<dim3(tiles, 1, (nzt + 3) / 4), T::NT, 0, st>>>(a); break;
    case 2: k_back_dd<ZL, XM, 2><<<dim3(tiles, 1, (nzt + 1) / 2), T::NT, 0, st>>>(a); break;
    default: k_back_dd<ZL, XM, 1><<<dim3(tiles, 1, nzt), T::NT, 0, st>>>(a); break;
  }
}

template <bool XM>
static void back_dd_zl(int ZL, const DdAdjArgs& a, int nzt, cudaStream_t st) {
  switch (ZL) {
    case 8: back_dd_go<8, XM>(a, nzt, st); break;
    case 4: back_dd_go<4, XM>(a, nzt, st); break;
    case 2: back_dd_go<2, XM>(a, nzt, st); break;
    default: back_dd_go<1, XM>(a, nzt, st); break;
  }
}

template <int ZL>
static void ref_dd_go(const DdRefArgs& a, int nzt, cudaStream_t st) {
  using T = DdBackTile<ZL>;
  const int tiles = ((a.YN + T::LT - 1) / T::LT) * ((a.XN + T::KT - 1) / T::KT);
  switch (dd_nz(nzt, a.nzc)) {
    case 4: k_back_ref_dd<ZL, 4><<<dim3(tiles, 1, (nzt + 3) / 4), T::NT, 0, st>>>(a); break;
    case 2: k_back_ref_dd<ZL, 2><<<dim3(tiles, 1, (nzt + 1) / 2), T::NT, 0, st>>>(a); break;
    default: k_back_ref_dd<ZL, 1><<<dim3(tiles, 1, nzt), T::NT, 0, st>>>(a); break;
  }
}

int make_back_dd_args(const Plan& p, int back_mode, const float* w, const ViewGeom* vg, const double2* fc,
                      const int* order, const int* counts, int PN, const BackEpi& epi, DdAdjArgs* pass1,
                      DdAdjArgs* pass2, DdRefArgs* ref) {
  int zt0 = 0, nzt = 0;
  ztile_range(p, epi.zlo, epi.zhi, &zt0, &nzt);
  if (back_mode == DDFAN_BACK_REF) {
    DdRefArgs a{};
    a.q = reinterpret_cast<const float4*>(w); a.P4 = p.P4; a.vg = vg;
    a.PN = PN; a.U = p.U; a.Z = p.Z; a.XN = p.XN; a.YN = p.YN;
    a.ocx = p.ocx; a.ocy = p.ocy; a.dx = p.dx;
    a.inv_sid = p.inv_sid; a.inv_dbeta = p.inv_dbeta; a.cnt = (double)p.detCntIdx + 0.5;
    a.epi = epi;
    a.zt0 = zt0;
    a.nzt = nzt;
    a.nzc = p.NZ;
    *ref = a;
    return nzt;
  }
  DdAdjArgs a{};
  a.w = reinterpret_cast<const float4*>(w); a.P4 = p.P4;
  a.vg = vg; a.fc = fc; a.tb = p.d_tb; a.lut = p.d_lut;
  a.order = order; a.counts = counts;
  a.t0 = p.t0; a.invdt = p.invdt; a.dirt = p.dirt; a.M = p.M;
  a.PN = PN; a.U = p.U; a.Z = p.Z; a.XN = p.XN; a.YN = p.YN;
  a.ocx = p.ocx; a.ocy = p.ocy; a.dx = p.dx;
  a.zt0 = zt0;
  a.nzt = nzt;
  a.nzc = p.NZ;
  // pass 1: x-major views along x columns -> tmp (mask applied)
  *pass1 = a;
  pass1->epi = epi;
  pass1->epi.out = p.d_tmp; pass1->epi.addend = nullptr; pass1->epi.xin = nullptr; pass1->epi.colsum = nullptr;
  pass1->epi.nonneg = 0;
  // pass 2: y-major views along y rows, plus pass 1, then the final epilogue
  *pass2 = a;
  pass2->epi = epi;
  pass2->epi.addend = p.d_tmp;
  return nzt;
}

int check_back_dd(const Plan& p, int back_mode, const int* order, const int* counts) {
  if (back_mode == DDFAN_BACK_REF) return DDFAN_OK;
  if (back_mode != DDFAN_BACK_ADJ) return set_err(DDFAN_ERR_ARG, "back_mode %d", back_mode);
  if (!p.adj_ok) return set_err(DDFAN_ERR_UNSUPPORTED, "detector boundaries are not monotone as seen from the source");
  if (!order || !counts) return set_err(DDFAN_ERR_ARG, "exact adjoint needs the view order");
  if (p.U + 1 > 1024 || p.M > 4096) return set_err(DDFAN_ERR_UNSUPPORTED, "exact adjoint: %d channels", p.U);
  return DDFAN_OK;
}

int launch_back_dd(const Plan& p, int back_mode, const float* w, const ViewGeom* vg, const double2* fc,
                   const int* order, const int* counts, int PN, const BackEpi& epi, cudaStream_t st) {
  int rc = check_back_dd(p, back_mode, order, counts);
  if (rc) return rc;
  DdAdjArgs a1, a2;
  DdRefArgs ar;
  const int nzt = make_back_dd_args(p, back_mode, w, vg, fc, order, counts, PN, epi, &a1, &a2, &ar);
  if (nzt == 0 || PN < 1) return DDFAN_OK;
  if (back_mode == DDFAN_BACK_REF) {
    ProfScope ps(KIND_BACK_A, st);
    switch (p.ZL) {
      case 8: ref_dd_go<8>(ar, nzt, st); break;
      case 4: ref_dd_go<4>(ar, nzt, st); break;
      case 2: ref_dd_go<2>(ar, nzt, st); break;
      default: ref_dd_go<1>(ar, nzt, st); break;
    }
    return check_launch("k_back_ref_dd");
  }
  {
    ProfScope ps(KIND_BACK_A, st);
    back_dd_zl<true>(p.ZL, a1, nzt, st);
  }
  rc = check_launch("k_back_dd<x>");
  if (rc) return rc;
  {
    ProfScope ps(KIND_BACK_B, st);
    back_dd_zl<false>(p.ZL, a2, nzt, st);
  }
  return check_launch("k_back_dd<y>");
}

// ------------------------------------------------------------------ device API

int proj_dev_shared(Plan& p, const float* d_angs, int stride, int PN, const float* d_vol, float* d_prj,
                    int zlo, int zhi, cudaStream_t st) {
  int rc;
  if ((rc = launch_view_geom(p, d_angs, stride, PN, p.d_vg, p.d_fc, p.d_cvd, st))) return rc;
  if ((rc = launch_view_order(p.d_vg, PN, p.d_order, p.d_counts, st))) return rc;
  if (p.mode == SAT_DIRECT) {
    // the kernel reads 4-slice float4 runs of a masked image: stage the
    // caller's image unless it already is one
    const float* img = d_vol;
    if (p.has_mask || (p.Z & 3) || (reinterpret_cast<uintptr_t>(d_vol) & 15)) {
      if ((rc = launch_stage_image(d_vol, p.Z, p.has_mask ? p.d_mask : nullptr, p.d_tmp, 4 * p.P4,
                                   (size_t)p.XN * p.YN, st)))
        return rc;
      img = p.d_tmp;
    }
    rc = launch_fwd_dd(p, img, p.d_vg, p.d_fc, p.d_cvd, p.d_order, PN, d_prj, p.U, p.Z, zlo, zhi, nullptr, st);
    mark_use(p, st);
    return rc;
  }
  if ((rc = launch_sat_image(p, d_vol, st, zlo, zhi))) return rc;
  rc = launch_fwd(p, p.d_vg, p.d_fc, p.d_cvd, p.d_order, PN, d_prj, zlo, zhi, st);
  mark_use(p, st);
  return rc;
}

int back_dev_shared(Plan& p, const float* d_angs, int stride, int PN, const float* d_prj, float* d_vol,
                    int back_mode, int zlo, int zhi, cudaStream_t st) {
  int rc;
  if ((rc = launch_view_geom(p, d_angs, stride, PN, p.d_vg, p.d_fc, p.d_cvd, st))) return rc;
  if ((rc = launch_view_order(p.d_vg, PN, p.d_order, p.d_counts, st))) return rc;
  const bool adj = back_mode == DDFAN_BACK_ADJ;
  BackEpi e{};
  e.out = d_vol; e.mask = p.has_mask ? p.d_mask : nullptr; e.zlo = zlo; e.zhi = zhi;
  if (p.mode == SAT_DIRECT) {
    float* w = reinterpret_cast<float*>(p.d_satq);
    if ((rc = launch_stage_sino(d_prj, p.Z, adj ? p.d_cvd : nullptr, p.U, w, 4 * p.P4, (size_t)PN, st))) return rc;
    rc = launch_back_dd(p, back_mode, w, p.d_vg, p.d_fc, p.d_order, p.d_counts, PN, e, st);
    mark_use(p, st);
    return rc;
  }
  if ((rc = launch_sat_sino(p, d_prj, PN, adj ? p.d_cvd : nullptr, 1.f, nullptr, nullptr, nullptr, st, zlo,
                            zhi)))
    return rc;
  rc = launch_back(p, back_mode, p.d_vg, p.d_fc, p.d_order, p.d_counts, PN, e, st);
  mark_use(p, st);
  return rc;
}

// Groups of slices sharing one angle list: per-slice angle arrays
// (hangs[PN][SLN]) become one launch per distinct list.
static void angle_groups(const float* hangs, int PN, int SLN, std::vector<std::vector<int>>& groups) {
  groups.clear();
  std::vector<int> rep;  // representative slice per group
  for (int z = 0; z < SLN; ++z) {
    int gi = -1;
    for (size_t g = 0; g < rep.size() && gi < 0; ++g) {
      const int r = rep[g];
      bool same = true;
      for (int q = 0; q < PN && same; ++q)
        same = std::memcmp(&hangs[(size_t)q * SLN + z], &hangs[(size_t)q * SLN + r], sizeof(float)) == 0;
      if (same) gi = (int)g;
    }
    if (gi < 0) {
      rep.push_back(z);
      groups.push_back({z});
    } else {
      groups[gi].push_back(z);
    }
  }
}

// Run `fn(angles-of-group, zlo, zhi)` once per group of slices with a common
// angle list; slices outside [zlo, zhi) are computed but not written.
template <class F>
static int for_angle_groups(Plan& p, const float* h_angs, int PN, F&& fn, cudaStream_t st) {
  std::vector<std::vector<int>> groups;
  angle_groups(h_angs, PN, p.Z, groups);
  std::vector<float> a(PN);
  for (auto& g : groups) {
    for (int q = 0; q < PN; ++q) a[q] = h_angs[(size_t)q * p.Z + g[0]];
    cudaError_t e = cudaMemcpyAsync(p.d_angs, a.data(), sizeof(float) * PN, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "angles upload: %s", cudaGetErrorString(e));
    // contiguous runs of the group
    size_t i = 0;
    while (i < g.size()) {
      size_t j = i + 1;
      while (j < g.size() && g[j] == g[j - 1] + 1) ++j;
      int rc = fn(p.d_angs, g[i], g[j - 1] + 1);
      if (rc) return rc;
      i = j;
    }
    // the pageable source buffer `a` is reused: make the copy complete first
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
  }
  return DDFAN_OK;
}

// ------------------------------------------------------------------ per-slice lists

// Slices the grouped path computes for these groups: every contiguous run of
// a group's slices costs the whole z-tiles that hold it.
static long long grouped_slices(const Plan& p, const std::vector<std::vector<int>>& groups) {
  const int tile = 4 * p.ZL;
  long long n = 0;
  for (auto& g : groups) {
    size_t i = 0;
    while (i < g.size()) {
      size_t j = i + 1;
      while (j < g.size() && g[j] == g[j - 1] + 1) ++j;
      n += (long long)((g[j - 1] + tile) / tile - g[i] / tile) * tile;
      i = j;
    }
  }
  return n;
}

// Time per slice of the slice-major kernels over the shared-list ones,
// measured at 512 x 512, 96 views: forward 1.45x, exact adjoint 2.7x, REF
// backprojector 4.4x (its FP64 geometry per sample is no longer shared by 32
// slices).  The grouped path costs its computed slices over Z times the
// shared-list time.
static bool use_slice_major(const Plan& p, const std::vector<std::vector<int>>& groups, int PN, double ratio) {
  return groups.size() > 1 && PN <= 65535 && (double)grouped_slices(p, groups) > ratio * p.Z;
}

static int ps_alloc(Plan& p) {
  if (p.ps_tabx) return DDFAN_OK;
  const size_t Z = (size_t)p.Z, R = Z * p.PNmax, U = (size_t)p.U;
  const size_t V = (size_t)p.XN * p.YN * Z, VG = (size_t)(p.XN + 2) * (p.YN + 2) * Z;
  const size_t CF = p.mode == SAT_FP32 ? 2 : 4;  // floats per slice-major cell
  size_t& B = p.bytes;
  cudaStream_t as = p.alloc_stream;
  int rc;
  const size_t B0 = B;
  if ((rc = dalloc(&p.ps_ang, R, &B, as)) || (rc = dalloc(&p.ps_vg, R, &B, as)) ||
      (rc = dalloc(&p.ps_fc, R * (U + 1), &B, as)) || (rc = dalloc(&p.ps_cvd, R * U, &B, as)) ||
      (rc = dalloc(&p.ps_img, V, &B, as)) || (rc = dalloc(&p.ps_imgt, V, &B, as)) ||
      (rc = dalloc(&p.ps_sino, R * U, &B, as)) || (rc = dalloc(&p.ps_tabx, CF * VG, &B, as)) ||
      (rc = dalloc(&p.ps_taby, CF * VG, &B, as)) || (rc = dalloc(&p.ps_sq, CF * R * (U + 1), &B, as))) {
    // release what was taken, so that a later call starts from nothing
    void** bufs[] = {(void**)&p.ps_ang, (void**)&p.ps_vg, (void**)&p.ps_fc, (void**)&p.ps_cvd,
                     (void**)&p.ps_img, (void**)&p.ps_imgt, (void**)&p.ps_sino, (void**)&p.ps_tabx,
                     (void**)&p.ps_taby, (void**)&p.ps_sq};
    for (void** q : bufs) {
      dev_free(*q, as);
      *q = nullptr;
    }
    B = B0;
    return rc;
  }
  // the allocations complete before any stream uses them
  cudaError_t e = cudaStreamSynchronize(as);
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "slice-major buffers: %s", cudaGetErrorString(e));
  return DDFAN_OK;
}

// geometry rows (z, m) of angle list d_angs [PN][Z]
static int ps_geometry(Plan& p, const float* d_angs, int PN, cudaStream_t st) {
  int rc = ps_transpose(d_angs, p.ps_ang, 1, PN, p.Z, st);
  if (rc) return rc;
  return launch_view_geom(p, p.ps_ang, 1, PN * p.Z, p.ps_vg, p.ps_fc, p.ps_cvd, st);
}

static int ps_proj_dev(Plan& p, const float* d_angs, int PN, const float* d_vol, float* d_prj, cudaStream_t st) {
  int rc;
  if ((rc = ps_alloc(p)) || (rc = ps_geometry(p, d_angs, PN, st))) return rc;
  const int Z = p.Z;
  {
    ProfScope ps(KIND_SAT_IMAGE, st);
    if ((rc = ps_transpose(d_vol, p.ps_img, 1, (long long)p.XN * p.YN, Z, st)) ||
        (rc = ps_transpose(p.ps_img, p.ps_imgt, Z, p.YN, p.XN, st)))
      return rc;
    PsScanArgs a{};
    a.mask = p.has_mask ? p.d_mask : nullptr;
    a.XN = p.XN; a.pad = 1;
    a.tab = p.ps_tabx; a.nlines = Z * p.YN; a.N = p.XN; a.Nw = p.XN + 2; a.src = p.ps_img; a.lines_per_slice = p.YN;
    if ((rc = ps_scan(p.mode, 0, a, st))) return rc;
    a.tab = p.ps_taby; a.nlines = Z * p.XN; a.N = p.YN; a.Nw = p.YN + 2; a.src = p.ps_imgt; a.lines_per_slice = p.XN;
    a.cols = 1;
    if ((rc = ps_scan(p.mode, 0, a, st))) return rc;
  }
  PsFwdArgs f;
  f.tabx = p.ps_tabx; f.taby = p.ps_taby; f.vg = p.ps_vg; f.fc = p.ps_fc; f.cvd = p.ps_cvd;
  f.out = p.ps_sino; f.cstride = PN; f.U = p.U; f.XN = p.XN; f.YN = p.YN; f.dx = (float)p.dx;
  if ((rc = ps_fwd(p.mode, f, PN, Z, st))) return rc;
  rc = ps_transpose(p.ps_sino, d_prj, 1, Z, PN * p.U, st);
  mark_use(p, st);
  return rc;
}

static int ps_back_dev(Plan& p, const float* d_angs, int PN, const float* d_prj, float* d_vol, int back_mode,
                       cudaStream_t st) {
  const bool adj = back_mode == DDFAN_BACK_ADJ;
  if (adj && !p.adj_ok) return set_err(DDFAN_ERR_UNSUPPORTED, "detector boundaries are not monotone as seen from the source");
  int rc;
  if ((rc = ps_alloc(p)) || (rc = ps_geometry(p, d_angs, PN, st))) return rc;
  const int Z = p.Z;
  {
    // channel prefix sums of every (slice, view) line, weighted for the exact adjoint
    ProfScope ps(KIND_SAT_SINO, st);
    if ((rc = ps_transpose(d_prj, p.ps_sino, 1, (long long)PN * p.U, Z, st))) return rc;
    PsScanArgs a{};
    a.tab = p.ps_sq; a.nlines = Z * PN; a.N = p.U; a.Nw = p.U + 1; a.src = p.ps_sino; a.lines_per_slice = 1;
    a.wgt = adj ? p.ps_cvd : nullptr; a.wscale = 1.f;
    if ((rc = ps_scan(p.mode, adj ? 2 : 0, a, st))) return rc;
  }
  PsBackArgs b{};
  b.sq = p.ps_sq; b.vg = p.ps_vg; b.fc = p.ps_fc;
  b.tb = p.d_tb; b.lut = p.d_lut; b.t0 = p.t0; b.invdt = p.invdt; b.dirt = p.dirt; b.M = p.M;
  b.cnt = PN; b.cstride = PN; b.U = p.U; b.XN = p.XN; b.YN = p.YN;
  b.ocx = p.ocx; b.ocy = p.ocy; b.dx = p.dx;
  b.inv_sid = p.inv_sid; b.inv_dbeta = p.inv_dbeta; b.cnt_ref = (double)p.detCntIdx + 0.5;
  b.out = p.ps_img; b.mask = p.has_mask ? p.d_mask : nullptr;
  if ((rc = adj ? ps_back(p.mode, b, Z, st) : ps_back_ref(p.mode, b, Z, st))) return rc;
  rc = ps_transpose(p.ps_img, d_vol, 1, Z, p.XN * p.YN, st);
  mark_use(p, st);
  return rc;
}

int proj_dev_per_slice(Plan& p, const float* d_angs, const float* h_angs, int PN, const float* d_vol,
                       float* d_prj, cudaStream_t st) {
  std::vector<std::vector<int>> groups;
  angle_groups(h_angs, PN, p.Z, groups);
  if (use_slice_major(p, groups, PN, 1.45)) return ps_proj_dev(p, d_angs, PN, d_vol, d_prj, st);
  return for_angle_groups(p, h_angs, PN, [&](const float* da, int zlo, int zhi) {
    return proj_dev_shared(p, da, 1, PN, d_vol, d_prj, zlo, zhi, st);
  }, st);
}

int back_dev_per_slice(Plan& p, const float* d_angs, const float* h_angs, int PN, const float* d_prj,
                       float* d_vol, int back_mode, cudaStream_t st) {
  std::vector<std::vector<int>> groups;
  angle_groups(h_angs, PN, p.Z, groups);
  if (use_slice_major(p, groups, PN, back_mode == DDFAN_BACK_ADJ ? 2.7 : 4.4))
    return ps_back_dev(p, d_angs, PN, d_prj, d_vol, back_mode, st);
  return for_angle_groups(p, h_angs, PN, [&](const float* da, int zlo, int zhi) {
    return back_dev_shared(p, da, 1, PN, d_prj, d_vol, back_mode, zlo, zhi, st);
  }, st);
}

}  // namespace ddfan

// ====================================================================== C ABI

using namespace ddfan;

extern "C" {

DDFAN_API const char* ddfan_last_error(void) { return ddfan::last_error(); }
DDFAN_API int ddfan_version(void) { return 1; }

DDFAN_API int ddfan_tune_set_zl(int zblocks, int zl) {
  if (zblocks < 1 || !(zl == 0 || zl == 1 || zl == 2 || zl == 4 || zl == 8) || zl > zblocks)
    return set_err(DDFAN_ERR_ARG, "tune_set_zl: zblocks=%d zl=%d", zblocks, zl);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  if (zl == 0) g_tuned_zl.erase(zblocks);
  else g_tuned_zl[zblocks] = zl;
  return DDFAN_OK;
}

DDFAN_API int ddfan_tune_get_zl(int zblocks) { return zblocks < 1 ? 0 : pow2_zl(zblocks); }

DDFAN_API int ddfan_tune_set_nz(int zblocks, int nz) {
  if (zblocks < 1 || !(nz == 0 || nz == 1 || nz == 2 || nz == 4))
    return set_err(DDFAN_ERR_ARG, "tune_set_nz: zblocks=%d nz=%d", zblocks, nz);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  if (nz == 0) g_tuned_nz.erase(zblocks);
  else g_tuned_nz[zblocks] = nz;
  return DDFAN_OK;
}

DDFAN_API int ddfan_tune_get_nz(int zblocks) { return zblocks < 1 ? 0 : plan_nz(zblocks); }

DDFAN_API size_t ddfan_plan_estimate_bytes(int XN, int YN, int DNU, int SLN, int PNmax, int sat_mode) {
  if (XN < 1 || YN < 1 || DNU < 2 || SLN < 1 || PNmax < 1 || sat_mode < 0 || sat_mode > SAT_DIRECT) return 0;
  const int P4 = (SLN + 3) / 4;
  int ZB = P4;
  const int ZL = pow2_zl(ZB);
  ZB = (ZB + ZL - 1) / ZL * ZL;
  const size_t F4 = cell_f4(sat_mode), U = (size_t)DNU, P = (size_t)PNmax;
  const bool direct = sat_mode == SAT_DIRECT;
  const size_t cells = direct ? P * (U + 1) * P4 : 2 * (size_t)XN * YN * ZB * F4 + P * (U + 1) * ZB * F4;
  const size_t tmp = (size_t)XN * YN * (direct ? 4 * (size_t)P4 : (size_t)SLN);
  return cells * sizeof(float4) + (2 * (U + 1) + 2 * U) * sizeof(double) + (size_t)XN * YN +
         (U + 1) * sizeof(float) + 4 * (U + 1) * sizeof(uint16_t) + P * sizeof(ViewGeom) +
         P * (U + 1) * sizeof(double2) + P * U * sizeof(float) + tmp * sizeof(float) +
         P * sizeof(float) + P * sizeof(int) + 2 * sizeof(int);
}

DDFAN_API int ddfan_fan_geometry(float sid, float sdd, int DNU, float detCellWidth, float detCntIdx,
                                 float* x0, float* y0, float* xds, float* yds) {
  if (DNU < 1 || !xds || !yds || !x0 || !y0) return set_err(DDFAN_ERR_ARG, "fan_geometry: bad arguments");
  // AAPM_script/DD2MutiSlices.m:55-76, in MATLAB single arithmetic
  const float stepTheta = atanf(detCellWidth / 2.0f / sdd) * 2.0f;
  for (int ii = 1; ii <= DNU; ++ii) {
    const float curBeta = ((float)ii - detCntIdx) * stepTheta;
    xds[ii - 1] = sinf(curBeta) * sdd;
    yds[ii - 1] = sid - cosf(curBeta) * sdd;
  }
  *x0 = 0.0f;
  *y0 = sid;
  return DDFAN_OK;
}

DDFAN_API int ddfan_plan_create(ddfan_plan** out, float x0, float y0, int DNU, const float* xds,
                                const float* yds, float detCntIdx, float imgXCenter, float imgYCenter,
                                int XN, int YN, float dx, const uint8_t* mask, int SLN, int PNmax,
                                int sat_mode, int device) {
  if (!out) return set_err(DDFAN_ERR_ARG, "out is null");
  PlanDesc d{x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, XN, YN, dx, mask, SLN, PNmax,
             sat_mode, device};
  Plan* p = nullptr;
  int rc = plan_create(&p, d);
  *out = reinterpret_cast<ddfan_plan*>(p);
  return rc;
}

DDFAN_API void ddfan_plan_destroy(ddfan_plan* plan) { plan_free(reinterpret_cast<Plan*>(plan)); }

DDFAN_API size_t ddfan_cached_bytes(int device) {
  cudaMemPool_t pool = lib_pool(device, false);
  if (!pool) return 0;
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return reserved > used ? (size_t)(reserved - used) : 0;
}

DDFAN_API int ddfan_release_cached(int device) {
  cudaMemPool_t pool = lib_pool(device, false);
  if (!pool) return DDFAN_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_ARG, "release_cached: device %d", device);
  }
  // blocks whose stream-ordered free has not completed yet are not unused
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "release_cached: %s", cudaGetErrorString(e));
  }
  return DDFAN_OK;
}

DDFAN_API size_t ddfan_plan_device_bytes(const ddfan_plan* plan) {
  return plan ? reinterpret_cast<const Plan*>(plan)->bytes : 0;
}

DDFAN_API int ddfan_proj_dev(ddfan_plan* plan, const float* d_angs, int PN, int angs_per_slice,
                             const float* d_vol, float* d_prj, void* stream) {
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (!p || !d_angs || !d_vol || !d_prj) return set_err(DDFAN_ERR_ARG, "proj_dev: null argument");
  if (PN < 1 || PN > p->PNmax) return set_err(DDFAN_ERR_ARG, "proj_dev: PN=%d outside [1, %d]", PN, p->PNmax);
  cudaStream_t st = (cudaStream_t)stream;
  DeviceGuard dg(p->device);
  if (!angs_per_slice) return proj_dev_shared(*p, d_angs, 1, PN, d_vol, d_prj, 0, p->Z, st);
  std::vector<float> h((size_t)PN * p->Z);
  cudaError_t e = cudaMemcpyAsync(h.data(), d_angs, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "angles download: %s", cudaGetErrorString(e));
  return proj_dev_per_slice(*p, d_angs, h.data(), PN, d_vol, d_prj, st);
}

DDFAN_API int ddfan_back_dev(ddfan_plan* plan, const float* d_angs, int PN, int angs_per_slice,
                             const float* d_prj, float* d_vol, int back_mode, void* stream) {
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (!p || !d_angs || !d_vol || !d_prj) return set_err(DDFAN_ERR_ARG, "back_dev: null argument");
  if (PN < 1 || PN > p->PNmax) return set_err(DDFAN_ERR_ARG, "back_dev: PN=%d outside [1, %d]", PN, p->PNmax);
  if (back_mode != DDFAN_BACK_REF && back_mode != DDFAN_BACK_ADJ)
    return set_err(DDFAN_ERR_ARG, "back_dev: back_mode %d", back_mode);
  cudaStream_t st = (cudaStream_t)stream;
  DeviceGuard dg(p->device);
  if (!angs_per_slice) return back_dev_shared(*p, d_angs, 1, PN, d_prj, d_vol, back_mode, 0, p->Z, st);
  std::vector<float> h((size_t)PN * p->Z);
  cudaError_t e = cudaMemcpyAsync(h.data(), d_angs, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "angles download: %s", cudaGetErrorString(e));
  return back_dev_per_slice(*p, d_angs, h.data(), PN, d_prj, d_vol, back_mode, st);
}

}  // extern "C"
