// ddfan_plan.h -- host-side plan object and internal launch functions of libddfan.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan_device.cuh"

namespace ddfan {

struct BackEpi;
struct DdFwdArgs;
struct DdAdjArgs;
struct DdRefArgs;

int set_err(int code, const char* fmt, ...);
const char* last_error();

struct PlanDesc {
  float x0, y0;
  int DNU;
  const float* xds;
  const float* yds;
  float detCntIdx, imgXCenter, imgYCenter;
  int XN, YN;
  float dx;
  const uint8_t* mask;
  int SLN, PNmax, sat_mode, device;
  int zl_force = 0;  // 1, 2, 4 or 8: exactly this many z-blocks per z-tile (else chosen by pow2_zl)
};

// Geometry and device scratch for one (image, detector, slice count) shape.
struct Plan {
  int device = 0;
  int XN = 0, YN = 0, U = 0, Z = 0, ZB = 0, PNmax = 0, mode = 0, ZL = 1;
  int P4 = 0;  // 4-slice blocks of the direct mode's operands: ceil(Z / 4)
  int NZ = 4;  // most z-tiles per thread of the direct kernels (1, 2 or 4)
  double x0 = 0, y0 = 0, dx = 1, ocx = 0, ocy = 0, detCntIdx = 0;
  double inv_dbeta = 0, inv_sid = 0;  // REF backprojector
  double sh0x = 0, sh0y = -1;         // unit vector source -> rotation centre, angle 0
  float t0 = 0, invdt = 0, dirt = 1;  // exact-adjoint bracket table
  int M = 0;
  bool adj_ok = true, has_mask = false;
  std::vector<double> bx, by;
  std::vector<float> xd, yd, tb;
  std::vector<uint16_t> lut;
  // device
  double *d_bx = nullptr, *d_by = nullptr, *d_xd = nullptr, *d_yd = nullptr;
  uint8_t* d_mask = nullptr;
  float* d_tb = nullptr;
  uint16_t* d_lut = nullptr;
  // prefix-sum tables; in the direct mode d_satq holds the staged sinogram
  // operand [PNmax][U+1][4 P4] and there are no image tables
  float4 *d_satx = nullptr, *d_saty = nullptr, *d_satq = nullptr;
  ViewGeom* d_vg = nullptr;
  double2* d_fc = nullptr;
  float* d_cvd = nullptr;
  float* d_tmp = nullptr;   // one image of scratch (exact adjoint, pass 1; the direct mode's staged image)
  float* d_angs = nullptr;  // PNmax angles (host-angle entry points)
  int* d_order = nullptr;   // PNmax views in dispatch order (x-major first)
  int* d_counts = nullptr;  // {x-major views, others}
  // slice-major buffers for per-slice angle lists (allocated on first use):
  // geometry rows z * PNmax + m, image [Z][YN][XN] and [Z][XN][YN], sinogram
  // [Z][PNmax][U], cell tables
  float* ps_ang = nullptr;
  ViewGeom* ps_vg = nullptr;
  double2* ps_fc = nullptr;
  float *ps_cvd = nullptr, *ps_img = nullptr, *ps_imgt = nullptr, *ps_sino = nullptr;
  float *ps_tabx = nullptr, *ps_taby = nullptr, *ps_sq = nullptr;
  cudaStream_t alloc_stream = nullptr;  // stream-ordered allocation / release
  cudaEvent_t last_use = nullptr;       // recorded after every call's launches
  size_t bytes = 0;
};

int plan_create(Plan** out, const PlanDesc& d);
// stream-ordered device allocation (never synchronises the device)
int dev_alloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);
// records the plan's last use on `st`; plan_free releases memory after it
void mark_use(Plan& p, cudaStream_t st);
// z-blocks per z-tile for a stack of ZB 4-slice blocks
int pow2_zl(int ZB);
// the z-tile width a plan uses: pow2_zl, narrowed by the DDFAN_ZL environment
// variable (1, 2, 4 or 8), or exactly zl_force when that is one of those
int plan_zl(int ZB, int zl_force);
// most z-tiles per thread of the direct kernels for a stack of ZB blocks
// (1, 2 or 4): the autotuner's record (ddfan_tune_set_nz), else 4
int plan_nz(int ZB);
// allows the direct forward kernels their dynamic shared memory on the
// current device (dev names it in an error); before any launch there
int dd_prepare_device(int dev);
// DD3Boundaries (AAPM_script/utilities.cuh:268-287), float-rounded like the reference stores them
void boundaries(int n, const float* c, std::vector<double>& out);
void plan_free(Plan* p);

int launch_view_geom(const Plan& p, const float* d_angs, int stride, int PN, ViewGeom* vg,
                     double2* fc, float* cvd, cudaStream_t st);
// Per-slice angle lists d_angs [PN][Z] (h_angs: the same on the host): one
// launch group per distinct list, or the slice-major kernels when groups would
// recompute many slices (exact adjoint and forward only).
int proj_dev_per_slice(Plan& p, const float* d_angs, const float* h_angs, int PN, const float* d_vol,
                       float* d_prj, cudaStream_t st);
int back_dev_per_slice(Plan& p, const float* d_angs, const float* h_angs, int PN, const float* d_prj,
                       float* d_vol, int back_mode, cudaStream_t st);
// The prefix-sum builders, the forward projector and the backprojector run
// only the z-blocks / z-tiles that hold slices [zlo, zhi) (zhi < 0: all);
// slices outside the range that share a block are computed but not written
// by the projectors.
int launch_sat_image(const Plan& p, const float* d_vol, cudaStream_t st, int zlo = 0, int zhi = -1);
// Per-slice view angles in the solver: each z-tile projects its own range of
// geometry rows (ztd[zt] = {first row, count, slot-order offset, x-major
// count}); row r is raw view r / Mc + (r % Mc) * nOS and slice z of the
// sinogram y reads that raw view as its view (raw view - soff[z]) of T, in
// subset ksub.  PN of the launches is then the largest count.
struct ViewRanges {
  const int4* ztd = nullptr;
  const int* soff = nullptr;
  int Mc = 1, nOS = 1, ksub = 0, T = 0;
};

int launch_sat_sino(const Plan& p, const float* d_prj, int PN, const float* wgt, float wscale,
                    const float* y, const int* yview, const float* rowsum, cudaStream_t st, int zlo = 0,
                    int zhi = -1, const ViewRanges* vr = nullptr);
int launch_fwd(const Plan& p, const ViewGeom* vg, const double2* fc, const float* cvd,
               const int* order, int PN, float* d_prj, int zlo, int zhi, cudaStream_t st,
               const int4* ztd = nullptr);
int launch_back(const Plan& p, int back_mode, const ViewGeom* vg, const double2* fc,
                const int* order, const int* counts, int PN, const BackEpi& epi, cudaStream_t st,
                const int4* ztd = nullptr);
int launch_view_order(const ViewGeom* vg, int PN, int* order, int* counts, cudaStream_t st);

// ---- direct mode (no prefix-sum tables; ddfan_dd_kernels.cuh)
// OS-SART residual fused into the forward projector's store: out = ((y - A x)
// / rowsum where rowsum != 0, else A x) * wgt (wgt null = 1).
struct DdResidual {
  const float* y = nullptr;       // measured [views][U][ystride]
  const int* yview = nullptr;     // slot -> measured view
  const float* rowsum = nullptr;  // [slot][U]
  const float* wgt = nullptr;     // [slot][U] or null
  int ystride = 0;
};
// Forward projection of the masked image img [YN][XN][4 P4] into
// out[slot][orow][ostride] (slices [zlo, zhi) written).
int launch_fwd_dd(const Plan& p, const float* img, const ViewGeom* vg, const double2* fc, const float* cvd,
                  const int* order, int PN, float* out, int orow, int ostride, int zlo, int zhi,
                  const DdResidual* res, cudaStream_t st);
// The arguments launch_fwd_dd would launch with (nzt: z-tiles of [zlo, zhi)).
DdFwdArgs make_fwd_dd_args(const Plan& p, const float* img, const ViewGeom* vg, const double2* fc,
                           const float* cvd, const int* order, int PN, float* out, int orow, int ostride, int zlo,
                           int zhi, const DdResidual* res);
// The arguments launch_back_dd would launch with: the exact adjoint's two
// passes, or the REF backprojector's one; returns the z-tile count.
int make_back_dd_args(const Plan& p, int back_mode, const float* w, const ViewGeom* vg, const double2* fc,
                      const int* order, const int* counts, int PN, const BackEpi& epi, DdAdjArgs* pass1,
                      DdAdjArgs* pass2, DdRefArgs* ref);
// what launch_back_dd checks before launching (status code)
int check_back_dd(const Plan& p, int back_mode, const int* order, const int* counts);
// Backprojection of w [slot][U+1][4 P4] (guard channel U = 0; weighted by
// 1/|dir.axis| for the exact adjoint) with the epilogue `epi`.
int launch_back_dd(const Plan& p, int back_mode, const float* w, const ViewGeom* vg, const double2* fc,
                   const int* order, const int* counts, int PN, const BackEpi& epi, cudaStream_t st);
// dst[pix][z < Zp] = z < Z ? src[pix][z] * mask : 0
int launch_stage_image(const float* src, int Z, const uint8_t* mask, float* dst, int Zp, size_t npix,
                       cudaStream_t st);
// dst[p][u <= U][z < Zp] = u < U && z < Z ? src[p][u][z] * wgt[p][u] : 0
int launch_stage_sino(const float* src, int Z, const float* wgt, int U, float* dst, int Zp, size_t PN,
                      cudaStream_t st);
// out[pix][z] = mask ? x[pix][z] : (clamp0 ? max(x0, 0) : x0)
int launch_publish_masked(const float* x, int Zi, const float* x0, int Z, const uint8_t* mask, int clamp0,
                          float* out, size_t npix, cudaStream_t st);
// k_view_order over nr ranges (desc[r] = {first row, count, order offset, -> x-major count})
int launch_view_order_ranges(const ViewGeom* vg, int4* desc, int nr, int* order, cudaStream_t st);
int proj_dev_shared(Plan& p, const float* d_angs, int stride, int PN, const float* d_vol,
                    float* d_prj, int zlo, int zhi, cudaStream_t st);
int back_dev_shared(Plan& p, const float* d_angs, int stride, int PN, const float* d_prj,
                    float* d_vol, int back_mode, int zlo, int zhi, cudaStream_t st);

// Optional per-launch CUDA-event profiler: when active on the calling thread,
// every kernel launch of the library is bracketed by two events on its stream.
enum LaunchKind {
  KIND_VIEW_GEOM = 0, KIND_SAT_IMAGE, KIND_FWD, KIND_SAT_SINO, KIND_BACK_A, KIND_BACK_B, KIND_FISTA,
  KIND_COUNT
};
struct LaunchProfiler {
  std::vector<cudaEvent_t> ev;  // pairs: before, after
  std::vector<int> kind;
  int mark(int k, cudaStream_t st);   // records the "before" event, returns the slot
  void done(int slot, cudaStream_t st);
  ~LaunchProfiler();
};
LaunchProfiler*& active_profiler();

// Brackets one launch with profiler events when a profiler is active.
struct ProfScope {
  LaunchProfiler* p;
  cudaStream_t st;
  int slot = -1;
  ProfScope(int kind, cudaStream_t s) : p(active_profiler()), st(s) {
    if (p) slot = p->mark(kind, st);
  }
  ~ProfScope() {
    if (p && slot >= 0) p->done(slot, st);
  }
};

// Makes `dev` current for the scope and restores the caller's device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace ddfan
