// ddfan_solver.cu -- mex-compatible host entry points and the device-resident
// OS-SART / FISTA solver of libddfan.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_kernels.cuh"
#include "ddfan_plan.h"

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

// Distinct angle lists among the slices of hangs[PN][SLN] (bitwise equal
// columns): slice_list[z] = list of slice z, rep[l] = first slice of list l.
void angle_lists(const float* hangs, int PN, int SLN, std::vector<int>& slice_list, std::vector<int>& rep) {
  std::vector<uint64_t> h(SLN, 1469598103934665603ull);
  for (int q = 0; q < PN; ++q) {
    const uint32_t* row = reinterpret_cast<const uint32_t*>(hangs + (size_t)q * SLN);
    for (int z = 0; z < SLN; ++z) h[z] = (h[z] ^ row[z]) * 1099511628211ull;
  }
  std::unordered_map<uint64_t, std::vector<int>> by_hash;
  slice_list.assign(SLN, -1);
  rep.clear();
  for (int z = 0; z < SLN; ++z) {
    std::vector<int>& cand = by_hash[h[z]];
    for (int l : cand) {
      bool same = true;
      for (int q = 0; q < PN && same; ++q)
        same = std::memcmp(&hangs[(size_t)q * SLN + z], &hangs[(size_t)q * SLN + rep[l]], sizeof(float)) == 0;
      if (same) {
        slice_list[z] = l;
        break;
      }
    }
    if (slice_list[z] < 0) {
      slice_list[z] = (int)rep.size();
      cand.push_back((int)rep.size());
      rep.push_back(z);
    }
  }
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
// (one launch group per distinct angle list), download.
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
  // per-slice angle lists: one launch group per distinct list
  std::vector<int> rep;
  std::vector<std::vector<int>> grp;
  for (int z = 0; z < p.Z; ++z) {
    int gi = -1;
    for (size_t k = 0; k < rep.size() && gi < 0; ++k) {
      bool same = true;
      for (int q = 0; q < PN && same; ++q)
        same = std::memcmp(&angs[(size_t)q * p.Z + z], &angs[(size_t)q * p.Z + rep[k]], sizeof(float)) == 0;
      if (same) gi = (int)k;
    }
    if (gi < 0) { rep.push_back(z); grp.push_back({z}); }
    else grp[gi].push_back(z);
  }
  std::vector<float> a(PN);
  for (auto& gr : grp) {
    for (int q = 0; q < PN; ++q) a[q] = angs[(size_t)q * p.Z + gr[0]];
    DDFAN_CK(cudaMemcpy(p.d_angs, a.data(), sizeof(float) * PN, cudaMemcpyHostToDevice));
    size_t i = 0;
    while (i < gr.size()) {
      size_t j = i + 1;
      while (j < gr.size() && gr[j] == gr[j - 1] + 1) ++j;
      rc = forward ? proj_dev_shared(p, p.d_angs, 1, PN, din.p, dout.p, gr[i], gr[j - 1] + 1, 0)
                   : back_dev_shared(p, p.d_angs, 1, PN, din.p, dout.p, back_mode, gr[i], gr[j - 1] + 1, 0);
      if (rc) return rc;
      i = j;
    }
    DDFAN_CK(cudaDeviceSynchronize());
  }
  DDFAN_CK(cudaMemcpy(out, dout.p, sizeof(float) * (forward ? S : V), cudaMemcpyDeviceToHost));
  return DDFAN_OK;
}

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
  for (size_t k = 0; k < slabs.size(); ++k) {
    const int a = slabs[k].first, b = slabs[k].second, n = b - a;
    PlanDesc d{x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, XN, YN, dx, mask, n, PN,
               sat_mode, (int)(k % ndev)};
    if (n == SLN) {
      rc = mex_slab(forward, d, hangs, PN, in, out, back_mode);
    } else {
      std::vector<float> sin, sang, sout(forward ? nray * n : npix * n);
      gather_slab(in, forward ? npix : nray, SLN, a, b, sin);
      gather_slab(hangs, PN, SLN, a, b, sang);
      rc = mex_slab(forward, d, sang.data(), PN, sin.data(), sout.data(), back_mode);
      if (!rc) scatter_slab(sout, forward ? nray : npix, SLN, a, b, out);
    }
    if (rc) return rc;
  }
  return DDFAN_OK;
}

// ====================================================================== solver

// Slices [z0, z1) whose angle lists are all list `list`.
struct Segment {
  int z0, z1, list;
};

struct Solver {
  Plan* P = nullptr;  // SLN slices, PNmax = largest subset
  int device = 0;
  int PNall = 0, nsub = 1, useFISTA = 1, nonneg = 0, back_mode = DDFAN_BACK_REF;
  int XN = 0, YN = 0, U = 0, Z = 0;
  std::vector<int> off, cnt;  // subset k: rows [off[k], off[k] + cnt[k]) of the subset-ordered tables
  // Distinct per-slice angle lists (hangs[PNall][SLN] columns): one set of
  // view tables per list, PNall rows each; runs of consecutive slices with one
  // list are segments, projected and backprojected by their own launches.
  int nlists = 1;
  std::vector<Segment> segs;
  ViewGeom* d_vg = nullptr;  // [nlists][PNall], subset order
  double2* d_fc = nullptr;   // [nlists][PNall][U+1]
  float* d_cvd = nullptr;    // [nlists][PNall][U]
  int* d_yview = nullptr;  // subset-ordered row -> original view index
  int* d_order = nullptr;  // [nlists][PNall]: per subset, views in dispatch order (x-major first)
  int* d_counts = nullptr; // [nlists][nsub][2]: per subset, {x-major views, others}
  float* d_rows = nullptr; // [PNall][U]   row sums, subset order
  float* d_cols = nullptr; // [nsub][YN][XN] column sums
  float* d_y = nullptr;    // [PNall][U][Z] measured sinogram, original order
  float* d_x = nullptr;
  float* d_xprev = nullptr;
  float* d_ax = nullptr;   // [PNmax][U][Z]
  double* d_t = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t last_use = nullptr;  // recorded after work enqueued on a caller's stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  size_t bytes = 0;
  int launches = 0;
};

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
                  s->d_y, s->d_x, s->d_xprev, s->d_ax, s->d_t};
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

// One OS-SART iteration (AAPM_script/OSSART_AAPM.m:79-115) on stream st.
// Segments run one after another: slices of a neighbouring segment that share
// a z-block are computed by each segment's launches but written only by their
// own, and each segment rebuilds the sinogram table it backprojects.
static int solver_iteration(Solver& s, cudaStream_t st) {
  Plan& p = *s.P;
  int rc, n = 0;
  const bool adj = s.back_mode == DDFAN_BACK_ADJ;
  const size_t P = (size_t)s.PNall;
  for (int k = 0; k < s.nsub; ++k) {
    const int o = s.off[k], c = s.cnt[k];
    // project the current image (:85)
    if ((rc = launch_sat_image(p, s.d_x, st))) return rc;
    ++n;
    for (const Segment& g : s.segs) {
      const size_t r = (size_t)g.list * P + o;
      const ViewGeom* vg = s.d_vg + r;
      const double2* fc = s.d_fc + r * (s.U + 1);
      const float* cvd = s.d_cvd + r * s.U;
      const int* order = s.d_order + r;
      if ((rc = launch_fwd(p, vg, fc, cvd, order, c, s.d_ax, g.z0, g.z1, st))) return rc;
      // residual (y - A x) / rowSum folded into the sinogram prefix sums (:86-88)
      if ((rc = launch_sat_sino(p, s.d_ax, c, adj ? cvd : nullptr, 1.f, s.d_y, s.d_yview + o,
                                s.d_rows + (size_t)o * s.U, st, g.z0, g.z1)))
        return rc;
      // backproject, divide by colSum, add, optional clamp (:91-97)
      BackEpi e{};
      e.out = s.d_x; e.xin = s.d_x; e.colsum = s.d_cols + (size_t)k * s.XN * s.YN;
      e.nonneg = s.nonneg; e.mask = p.has_mask ? p.d_mask : nullptr; e.zlo = g.z0; e.zhi = g.z1;
      const int* counts = s.d_counts + ((size_t)g.list * s.nsub + k) * 2;
      if ((rc = launch_back(p, s.back_mode, vg, fc, order, counts, c, e, st))) return rc;
      n += adj ? 4 : 3;
    }
  }
  if (s.useFISTA) {
    const size_t V = (size_t)s.XN * s.YN * s.Z;
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
  // distinct angle lists (bitwise) and the slices' runs of them
  std::vector<int> rep, slice_list(SLN);
  angle_lists(hangs, PNall, SLN, slice_list, rep);
  s.nlists = (int)rep.size();
  int shortest = SLN;
  for (int z = 0; z < SLN;) {
    int e = z + 1;
    while (e < SLN && slice_list[e] == slice_list[z]) ++e;
    s.segs.push_back({z, e, slice_list[z]});
    shortest = std::min(shortest, e - z);
    z = e;
  }
  // subsets k, k + numOfOS, ... (AAPM_script/OSSART_AAPM.m:60)
  std::vector<int> yview;
  int PNmax = 0;
  for (int k = 0; k < numOfOS; ++k) {
    s.off.push_back((int)yview.size());
    for (int v = k; v < PNall; v += numOfOS) yview.push_back(v);
    s.cnt.push_back((int)yview.size() - s.off.back());
    PNmax = std::max(PNmax, s.cnt.back());
  }
  const size_t P = (size_t)PNall, L = (size_t)s.nlists;
  std::vector<float> angs(L * P);
  for (size_t l = 0; l < L; ++l)
    for (size_t r = 0; r < P; ++r) angs[l * P + r] = hangs[(size_t)yview[r] * SLN + rep[l]];
  PlanDesc d{x0, y0, DNU, xds, yds, detCntIdx, imgXCenter, imgYCenter, XN, YN, dx, mask, SLN, PNmax,
             sat_mode, device};
  // z-tiles no wider than the shortest segment (a launch computes whole tiles)
  if (s.segs.size() > 1) d.zl_cap = std::max(1, std::min(8, shortest / 4));
  int rc = plan_create(&s.P, d);
  if (rc) return rc;
  s.bytes = s.P->bytes;
  DeviceGuard g(device);
  const size_t V = (size_t)XN * YN * SLN;
  DDFAN_CK(cudaStreamCreateWithFlags(&s.own, cudaStreamNonBlocking));
  DDFAN_CK(cudaEventCreateWithFlags(&s.last_use, cudaEventDisableTiming));
  if ((rc = salloc(s, &s.d_vg, L * P)) || (rc = salloc(s, &s.d_fc, L * P * (DNU + 1))) ||
      (rc = salloc(s, &s.d_cvd, L * P * DNU)) || (rc = salloc(s, &s.d_yview, PNall)) ||
      (rc = salloc(s, &s.d_order, L * P)) || (rc = salloc(s, &s.d_counts, L * 2 * (size_t)numOfOS)) ||
      (rc = salloc(s, &s.d_rows, (size_t)PNall * DNU)) ||
      (rc = salloc(s, &s.d_cols, (size_t)numOfOS * XN * YN)) ||
      (rc = salloc(s, &s.d_y, (size_t)PNall * DNU * SLN)) || (rc = salloc(s, &s.d_x, V)) ||
      (rc = salloc(s, &s.d_xprev, V)) || (rc = salloc(s, &s.d_ax, (size_t)PNmax * DNU * SLN)) ||
      (rc = salloc(s, &s.d_t, 1)))
    return rc;
  cudaStream_t st = s.own;
  // per-view tables for every view of every list, in subset order
  DevBuf<float> dang(st);
  if ((rc = dang.alloc(L * P))) return rc;
  DDFAN_CK(cudaMemcpyAsync(dang.p, angs.data(), sizeof(float) * L * P, cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemcpyAsync(s.d_yview, yview.data(), sizeof(int) * PNall, cudaMemcpyHostToDevice, st));
  if ((rc = launch_view_geom(*s.P, dang.p, 1, (int)(L * P), s.d_vg, s.d_fc, s.d_cvd, st))) return rc;
  // per list and subset: views of one orientation together (one image table
  // at a time stays hot in L2; the exact adjoint visits each orientation in turn)
  for (size_t l = 0; l < L; ++l)
    for (int k = 0; k < numOfOS; ++k)
      if ((rc = launch_view_order(s.d_vg + l * P + s.off[k], s.cnt[k], s.d_order + l * P + s.off[k],
                                  s.d_counts + (l * numOfOS + k) * 2, st)))
        return rc;
  // the weights use slice 0's angles (AAPM_script/OSSART_AAPM.m:61-64)
  const size_t l0 = (size_t)slice_list[0] * P;
  // row / column sums from slice 0 on a one-slice plan (AAPM_script/OSSART_AAPM.m:59-66)
  {
    PlanDesc d1 = d;
    d1.SLN = 1;
    PlanPtr P1;
    if ((rc = plan_create(&P1.p, d1))) return rc;
    DevBuf<float> ones(st), tmp(st);
    const size_t n1 = std::max((size_t)XN * YN, (size_t)PNmax * DNU);
    if ((rc = ones.alloc(n1)) || (rc = tmp.alloc((size_t)PNmax * DNU))) return rc;
    std::vector<float> h1(n1, 1.0f);
    DDFAN_CK(cudaMemcpyAsync(ones.p, h1.data(), sizeof(float) * n1, cudaMemcpyHostToDevice, st));
    if ((rc = launch_sat_image(*P1.p, ones.p, st))) return rc;
    for (int k = 0; k < numOfOS; ++k) {
      const size_t o = l0 + s.off[k];
      const int c = s.cnt[k];
      if ((rc = launch_fwd(*P1.p, s.d_vg + o, s.d_fc + o * (DNU + 1), s.d_cvd + o * DNU, s.d_order + o, c,
                           s.d_rows + (size_t)s.off[k] * DNU, 0, 1, st)))
        return rc;
    }
    for (int k = 0; k < numOfOS; ++k) {
      const size_t o = l0 + s.off[k];
      const int c = s.cnt[k];
      const bool adj = back_mode == DDFAN_BACK_ADJ;
      if ((rc = launch_sat_sino(*P1.p, ones.p, c, adj ? s.d_cvd + o * DNU : nullptr, 1.f, nullptr, nullptr,
                                nullptr, st)))
        return rc;
      BackEpi e{};
      e.out = s.d_cols + (size_t)k * XN * YN;
      e.mask = P1.p->has_mask ? P1.p->d_mask : nullptr;
      e.zlo = 0; e.zhi = 1;
      if ((rc = launch_back(*P1.p, back_mode, s.d_vg + o, s.d_fc + o * (DNU + 1), s.d_order + o,
                            s.d_counts + ((size_t)slice_list[0] * numOfOS + k) * 2, c, e, st)))
        return rc;
    }
    DDFAN_CK(cudaStreamSynchronize(st));
  }
  const double one = 1.0;
  DDFAN_CK(cudaMemcpyAsync(s.d_t, &one, sizeof(double), cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemsetAsync(s.d_x, 0, sizeof(float) * V, st));
  DDFAN_CK(cudaMemsetAsync(s.d_xprev, 0, sizeof(float) * V, st));
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
  const size_t U = (size_t)DNU, P = (size_t)PNall, V = (size_t)XN * YN * SLN;
  const size_t plan = ddfan_plan_estimate_bytes(XN, YN, DNU, SLN, (int)PNmax, sat_mode);
  if (!plan) return 0;
  const size_t own = P * sizeof(ViewGeom) + P * (U + 1) * sizeof(double2) + P * U * sizeof(float) +
                     3 * P * sizeof(int) + 2 * (size_t)numOfOS * sizeof(int) + P * U * sizeof(float) +
                     (size_t)numOfOS * XN * YN * sizeof(float) + P * U * SLN * sizeof(float) +
                     2 * V * sizeof(float) + PNmax * U * SLN * sizeof(float) + sizeof(double);
  // transient at creation: the one-slice weight plan and its buffers
  const size_t weights = ddfan_plan_estimate_bytes(XN, YN, DNU, 1, (int)PNmax, sat_mode) +
                         (std::max((size_t)XN * YN, PNmax * U) + PNmax * U + P) * sizeof(float);
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
  DDFAN_CK(cudaMemcpyAsync(s->d_y, proj, sizeof(float) * n,
                           is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           (cudaStream_t)stream));
  cudaEventRecord(s->last_use, (cudaStream_t)stream);
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_set_image(ddfan_ossart* h, const float* img, int is_device, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || !img) return set_err(DDFAN_ERR_ARG, "null argument");
  DeviceGuard g(s->device);
  const size_t n = (size_t)s->XN * s->YN * s->Z;
  cudaStream_t st = (cudaStream_t)stream;
  DDFAN_CK(cudaMemcpyAsync(s->d_x, img, sizeof(float) * n,
                           is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  DDFAN_CK(cudaMemcpyAsync(s->d_xprev, s->d_x, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
  static const double one = 1.0;
  DDFAN_CK(cudaMemcpyAsync(s->d_t, &one, sizeof(double), cudaMemcpyHostToDevice, st));
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
    }
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
  for (int it = 0; it < numOfIter; ++it) DDFAN_CK(cudaGraphLaunch(s->gexec, st));
  cudaEventRecord(s->last_use, st);
  return DDFAN_OK;
}

DDFAN_API int ddfan_ossart_get_image(ddfan_ossart* h, float* img, int is_device, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s || !img) return set_err(DDFAN_ERR_ARG, "null argument");
  DeviceGuard g(s->device);
  const size_t n = (size_t)s->XN * s->YN * s->Z;
  cudaStream_t st = (cudaStream_t)stream;
  DDFAN_CK(cudaMemcpyAsync(img, s->d_x, sizeof(float) * n,
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
  for (int it = 0; it < numOfIter && !rc; ++it) rc = solver_iteration(*s, st);
  active_profiler() = nullptr;
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
  return s ? s->d_x : nullptr;
}

DDFAN_API int ddfan_ossart_launches_per_iter(const ddfan_ossart* h) {
  const Solver* s = reinterpret_cast<const Solver*>(h);
  if (!s) return 0;
  const int per_seg = s->back_mode == DDFAN_BACK_ADJ ? 4 : 3;
  return s->nsub * (1 + (int)s->segs.size() * per_seg) + (s->useFISTA ? 2 : 0);
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
