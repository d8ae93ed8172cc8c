// ddfan_noalloc.cu -- forward projection that allocates no device memory.
//
// ddfan_proj_dev needs a plan, and a plan holds cudaMalloc'd prefix-sum and
// geometry tables.  Some callers cannot allocate: their device memory is
// owned up front by another allocator (a framework's caching allocator or a
// pool reserved at start-up), or they cannot afford cudaMalloc's implicit
// device-wide synchronisation in the middle of a pipeline.  For them,
// ddfan_proj_noalloc runs the same kernels with every scratch table placed
// in one file-scope device array of DDFAN_NOALLOC_SCRATCH_BYTES.  The array
// exists on every GPU that loads this library, for as long as it stays
// loaded.  Calls share it, so two calls whose kernels overlap on a GPU race
// on it: issue them on one stream, or order them.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>  // driver types only: the two driver calls go through cudaGetDriverEntryPoint
#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_kernels.cuh"
#include "ddfan_plan.h"

namespace ddfan {
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[DDFAN_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
void* g_addr[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 when unknown).  A
// device reset destroys the context that held the scratch array; the next
// context loads the array again, possibly at another address, under a new id.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Device address of the scratch array on `dev` (the current device).  In host
// code the array's name only stands in for it, so the set-up looks the
// address up with cudaGetSymbolAddress once per device -- again after a
// device reset, which gives the device a new context (when the context id
// cannot be read, on every call).
int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return set_err(DDFAN_ERR_UNSUPPORTED, "device index %d", dev);
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev] || ctx == 0 || ctx != g_ctx_id[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_err(DDFAN_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    }
    // the direct forward kernels' shared memory limit, set in this context too
    const int rc = dd_prepare_device(dev);
    if (rc) return rc;
    g_addr[dev] = p;
    // the lookup made the device's context current if none was
    g_ctx_id[dev] = current_context_id();
  }
  *out = static_cast<unsigned char*>(g_addr[dev]);
  return DDFAN_OK;
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }

}  // namespace
}  // namespace ddfan

using namespace ddfan;

extern "C" DDFAN_API int ddfan_proj_noalloc(float x0, float y0, int DNU, const float* xds,
                                            const float* yds, float imgXCenter, float imgYCenter,
                                            const float* d_angs, int PN, int XN, int YN, int SLN,
                                            const float* d_vol, float dx, const uint8_t* mask,
                                            int sat_mode, float* d_prj, void* stream) {
  if (!xds || !yds || !d_angs || !d_vol || !d_prj) return set_err(DDFAN_ERR_ARG, "proj_noalloc: null argument");
  if (DNU < 2 || XN < 1 || YN < 1 || SLN < 1 || PN < 1)
    return set_err(DDFAN_ERR_ARG, "proj_noalloc: bad sizes (DNU=%d XN=%d YN=%d SLN=%d PN=%d)", DNU, XN, YN,
                   SLN, PN);
  if (XN > 1024 || YN > 1024 || DNU + 1 > 1024)
    return set_err(DDFAN_ERR_UNSUPPORTED, "proj_noalloc: lines longer than 1024 cells are not supported");
  if (!(dx > 0.f)) return set_err(DDFAN_ERR_ARG, "proj_noalloc: dx must be > 0");
  if (sat_mode < SAT_FP32 || sat_mode > SAT_DIRECT)
    return set_err(DDFAN_ERR_ARG, "proj_noalloc: sat_mode %d", sat_mode);
  cudaStream_t st = (cudaStream_t)stream;
  // Every call uploads its geometry from host memory that is gone when the
  // call returns, so a call cannot be recorded into a graph: refuse one made
  // while its stream is being captured, before any other CUDA call.
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(DDFAN_ERR_CUDA, "proj_noalloc: stream query: %s", cudaGetErrorString(e));
    }
    if (cs != cudaStreamCaptureStatusNone)
      return set_err(DDFAN_ERR_UNSUPPORTED,
                     "proj_noalloc: the stream is being captured; this entry point uploads host geometry on "
                     "every call and does not run under stream capture");
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "proj_noalloc: no current CUDA device");
  }
  // a plan on the host stack whose device tables all point into the scratch array
  Plan p;
  p.device = dev;
  p.XN = XN; p.YN = YN; p.U = DNU; p.Z = SLN; p.ZB = (SLN + 3) / 4;
  p.PNmax = PN; p.mode = sat_mode; p.ZL = plan_zl(p.ZB, 0);  // the z-tile width a plan would take
  p.NZ = plan_nz(p.ZB);
  p.P4 = p.ZB;
  p.ZB = (p.ZB + p.ZL - 1) / p.ZL * p.ZL;
  p.x0 = x0; p.y0 = y0; p.dx = dx;
  p.ocx = (XN - 1.0) * 0.5 - (double)imgXCenter / (double)dx;
  p.ocy = (YN - 1.0) * 0.5 - (double)imgYCenter / (double)dx;
  boundaries(DNU, xds, p.bx);
  boundaries(DNU, yds, p.by);
  std::vector<double> xd(xds, xds + DNU), yd(yds, yds + DNU);
  // the mask goes through a pageable copy too: cudaMemcpyAsync has read it by
  // the time it returns, so the caller's buffer need not outlive the call
  std::vector<uint8_t> hmask;
  if (mask) hmask.assign(mask, mask + (size_t)XN * YN);
  p.has_mask = mask != nullptr;
  const bool direct = sat_mode == SAT_DIRECT;
  // the direct kernels read 4-slice float4 runs of a masked image: staged
  // unless the caller's image already is one
  const bool stage = direct && (mask || (SLN & 3) || (reinterpret_cast<uintptr_t>(d_vol) & 15));
  // Carve the scratch array.  Nothing in it needs to start at zero: each
  // region is written by this call before it is read, except the padding
  // z-blocks of the prefix-sum tables' last z-tile, which no kernel writes
  // and the forward projector reads only for slices past SLN, whose results
  // it drops -- a previous call's contents there are harmless.
  const size_t cells = direct ? 0 : (size_t)XN * YN * p.ZB * cell_f4(sat_mode);
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += align256(bytes); return o; };
  const size_t o_bx = take(sizeof(double) * (DNU + 1)), o_by = take(sizeof(double) * (DNU + 1));
  const size_t o_xd = take(sizeof(double) * DNU), o_yd = take(sizeof(double) * DNU);
  const size_t o_mask = take(mask ? (size_t)XN * YN : 0);
  const size_t o_vg = take(sizeof(ViewGeom) * PN), o_fc = take(sizeof(double2) * PN * (DNU + 1));
  const size_t o_cvd = take(sizeof(float) * PN * DNU), o_ord = take(sizeof(int) * PN);
  const size_t o_cnt = take(sizeof(int) * 2);
  const size_t o_satx = take(sizeof(float4) * cells), o_saty = take(sizeof(float4) * cells);
  const size_t o_img = take(stage ? sizeof(float4) * (size_t)XN * YN * p.P4 : 0);
  if (off > DDFAN_NOALLOC_SCRATCH_BYTES)
    return set_err(DDFAN_ERR_UNSUPPORTED,
                   "proj_noalloc: this problem needs %zu bytes of scratch, the fixed scratch array holds %llu "
                   "(use ddfan_plan_create + ddfan_proj_dev)",
                   off, (unsigned long long)DDFAN_NOALLOC_SCRATCH_BYTES);
  unsigned char* base = nullptr;
  int rc = scratch_address(dev, &base);
  if (rc) return rc;
  p.d_bx = reinterpret_cast<double*>(base + o_bx);
  p.d_by = reinterpret_cast<double*>(base + o_by);
  p.d_xd = reinterpret_cast<double*>(base + o_xd);
  p.d_yd = reinterpret_cast<double*>(base + o_yd);
  p.d_mask = mask ? base + o_mask : nullptr;
  p.d_vg = reinterpret_cast<ViewGeom*>(base + o_vg);
  p.d_fc = reinterpret_cast<double2*>(base + o_fc);
  p.d_cvd = reinterpret_cast<float*>(base + o_cvd);
  p.d_order = reinterpret_cast<int*>(base + o_ord);
  p.d_counts = reinterpret_cast<int*>(base + o_cnt);
  if (!direct) {
    p.d_satx = reinterpret_cast<float4*>(base + o_satx);
    p.d_saty = reinterpret_cast<float4*>(base + o_saty);
  }
  // host -> scratch copies of the small geometry arrays (pageable sources are
  // staged before cudaMemcpyAsync returns)
  cudaError_t e = cudaMemcpyAsync(p.d_bx, p.bx.data(), sizeof(double) * (DNU + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_by, p.by.data(), sizeof(double) * (DNU + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_xd, xd.data(), sizeof(double) * DNU, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p.d_yd, yd.data(), sizeof(double) * DNU, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && mask) e = cudaMemcpyAsync(p.d_mask, hmask.data(), hmask.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    p.d_bx = p.d_by = p.d_xd = p.d_yd = nullptr;
    return set_err(DDFAN_ERR_CUDA, "proj_noalloc: geometry upload: %s", cudaGetErrorString(e));
  }
  if (!(rc = launch_view_geom(p, d_angs, 1, PN, p.d_vg, p.d_fc, p.d_cvd, st)) &&
      !(rc = launch_view_order(p.d_vg, PN, p.d_order, p.d_counts, st))) {
    if (direct) {
      const float* img = d_vol;
      if (stage) {
        float* si = reinterpret_cast<float*>(base + o_img);
        rc = launch_stage_image(d_vol, SLN, p.d_mask, si, 4 * p.P4, (size_t)XN * YN, st);
        img = si;
      }
      if (!rc) rc = launch_fwd_dd(p, img, p.d_vg, p.d_fc, p.d_cvd, p.d_order, PN, d_prj, DNU, SLN, 0, SLN, nullptr, st);
    } else if (!(rc = launch_sat_image(p, d_vol, st))) {
      rc = launch_fwd(p, p.d_vg, p.d_fc, p.d_cvd, p.d_order, PN, d_prj, 0, SLN, st);
    }
  }
  // the stack plan does not own its device pointers
  p.d_bx = p.d_by = p.d_xd = p.d_yd = nullptr;
  return rc;
}
