// ddfan_batch.cu -- many OS-SART solves advanced together: one launch per
// kernel kind, subset step and tile class over a device work list of every
// solve's CTAs, instead of one launch per solve.
//
// A batched iteration runs subset step k of every solve that has one: the
// forward projectors (with the fused residual) of all those solves in one
// launch per (z-lane count, z-tiles per thread) class, then the
// backprojections the same way (the exact adjoint's x-column pass of every
// solve, then its y-row pass; or the reference backprojector), then FISTA of
// every solve in one launch pair.  Each CTA reads its item {solve's argument
// block, view row or voxel tile, channel block, z-tile group} and runs the
// same kernel body a single solve's launch runs, with that solve's arguments,
// so every solve computes exactly what it computes alone.  Small solves
// (a few slices, a few hundred views) that leave most of the GPU idle in a
// launch of their own fill it together.  The iteration is captured as one
// CUDA graph.  No counterpart in the reference, which runs one
// reconstruction per MATLAB call (AAPM_script/OSSART_AAPM.m:85, :92).
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_kernels.cuh"
#include "ddfan_plan.h"
#include "ddfan_solver.h"

namespace ddfan {

namespace {

enum BatchKind { BK_FWD = 0, BK_ADJ_X = 1, BK_ADJ_Y = 2, BK_REF = 3 };

struct BatchLaunch {
  int kind, ZL, NZ;
  size_t items_off, nitems;
  int group;  // the solver group whose chain the launch belongs to
};

int fwd_cw(int ZL, int NZ) {
  switch (ZL * 8 + NZ) {
    case 8 * 8 + 4: return DdFwdTile<8, DdFwdCG<8>::v, 4>::CW;
    case 8 * 8 + 2: return DdFwdTile<8, DdFwdCG<8>::v, 2>::CW;
    case 8 * 8 + 1: return DdFwdTile<8, DdFwdCG<8>::v, 1>::CW;
    case 4 * 8 + 4: return DdFwdTile<4, DdFwdCG<4>::v, 4>::CW;
    case 4 * 8 + 2: return DdFwdTile<4, DdFwdCG<4>::v, 2>::CW;
    case 4 * 8 + 1: return DdFwdTile<4, DdFwdCG<4>::v, 1>::CW;
    case 2 * 8 + 4: return DdFwdTile<2, DdFwdCG<2>::v, 4>::CW;
    case 2 * 8 + 2: return DdFwdTile<2, DdFwdCG<2>::v, 2>::CW;
    case 2 * 8 + 1: return DdFwdTile<2, DdFwdCG<2>::v, 1>::CW;
    case 1 * 8 + 4: return DdFwdTile<1, DdFwdCG<1>::v, 4>::CW;
    case 1 * 8 + 2: return DdFwdTile<1, DdFwdCG<1>::v, 2>::CW;
    default: return DdFwdTile<1, DdFwdCG<1>::v, 1>::CW;
  }
}

// (lines per tile, voxels per line per tile) of the direct exact adjoint and
// of the REF backprojector
void adj_tile(int ZL, int* LT, int* KT) {
  switch (ZL) {
    case 8: *LT = DdBackTile<8>::LT; *KT = DdBackTile<8>::KT; break;
    case 4: *LT = DdBackTile<4>::LT; *KT = DdBackTile<4>::KT; break;
    case 2: *LT = DdBackTile<2>::LT; *KT = DdBackTile<2>::KT; break;
    default: *LT = DdBackTile<1>::LT; *KT = DdBackTile<1>::KT; break;
  }
}

template <int ZL, int NZ>
void go_fwd(const DdFwdArgs* a, const int4* it, unsigned n, cudaStream_t st) {
  k_fwd_dd_batch<ZL, DdFwdCG<ZL>::v, NZ><<<n, 256, DdFwdTile<ZL, DdFwdCG<ZL>::v, NZ>::DYN, st>>>(a, it);
}

template <int ZL, int NZ>
void go_adj(bool xm, const DdAdjArgs* a, const int4* it, unsigned n, cudaStream_t st) {
  if (xm) k_back_dd_batch<ZL, true, NZ><<<n, 256, 0, st>>>(a, it);
  else k_back_dd_batch<ZL, false, NZ><<<n, 256, 0, st>>>(a, it);
}

template <int ZL, int NZ>
void go_ref(const DdRefArgs* a, const int4* it, unsigned n, cudaStream_t st) {
  k_back_ref_dd_batch<ZL, NZ><<<n, 256, 0, st>>>(a, it);
}

// solver groups whose launch chains run side by side (DDFAN_BATCH_GROUPS in
// the environment overrides it)
#ifndef DDFAN_BATCH_GROUPS
#define DDFAN_BATCH_GROUPS 1
#endif

// the work-list forward kernels' dynamic shared memory on the current device
// (at every batch creation: the attribute belongs to the context)
int batch_prepare_device(int dev) {
  cudaError_t e = cudaSuccess;
#define DDFAN_DD_ALLOW(ZLv, NZv)                                                                        \
  if (e == cudaSuccess)                                                                                 \
    e = dd_allow_dyn(k_fwd_dd_batch<ZLv, DdFwdCG<ZLv>::v, NZv>, DdFwdTile<ZLv, DdFwdCG<ZLv>::v, NZv>::DYN);
  DDFAN_DD_ALLOW(8, 4) DDFAN_DD_ALLOW(8, 2) DDFAN_DD_ALLOW(8, 1)
  DDFAN_DD_ALLOW(4, 4) DDFAN_DD_ALLOW(4, 2) DDFAN_DD_ALLOW(4, 1)
  DDFAN_DD_ALLOW(2, 4) DDFAN_DD_ALLOW(2, 2) DDFAN_DD_ALLOW(2, 1)
  DDFAN_DD_ALLOW(1, 4) DDFAN_DD_ALLOW(1, 2) DDFAN_DD_ALLOW(1, 1)
#undef DDFAN_DD_ALLOW
  if (e != cudaSuccess)
    return set_err(DDFAN_ERR_CUDA, "batched forward kernel attributes on device %d: %s", dev, cudaGetErrorString(e));
  return DDFAN_OK;
}

#define DDFAN_BATCH_ZL_NZ(ZLv, NZv, CALL) \
  if (L.ZL == ZLv && L.NZ == NZv) {       \
    CALL;                                 \
    break;                                \
  }

}  // namespace

struct Batch {
  int device = 0;
  std::vector<Solver*> sv;
  std::vector<BatchLaunch> launches;  // one iteration, in order
  DdFwdArgs* d_fargs = nullptr;
  DdAdjArgs* d_aargs = nullptr;
  DdRefArgs* d_rargs = nullptr;
  int4* d_items = nullptr;
  FistaDesc* d_fista = nullptr;
  int nfista = 0;
  size_t fista_max = 0;
  cudaStream_t own = nullptr;
  cudaEvent_t last_use = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int kernel_launches = 0;
  // side streams and events of the solver groups' chains (parallel branches
  // of the captured graph); group g's launches are contiguous in `launches`
  int groups = 1;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
};

static void batch_free(Batch* b) {
  if (!b) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  if (b->own && b->last_use) {
    cudaStreamWaitEvent(b->own, b->last_use, 0);
    cudaStreamSynchronize(b->own);
  }
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  void* ptrs[] = {b->d_fargs, b->d_aargs, b->d_rargs, b->d_items, b->d_fista};
  for (void* q : ptrs) dev_free(q, b->own);
  if (b->own) cudaStreamDestroy(b->own);
  if (b->last_use) cudaEventDestroy(b->last_use);
  for (cudaStream_t q : b->side) cudaStreamDestroy(q);
  for (cudaEvent_t q : b->join) cudaEventDestroy(q);
  if (b->fork) cudaEventDestroy(b->fork);
  cudaGetLastError();
  if (prev >= 0) cudaSetDevice(prev);
  delete b;
}

// One launch of the work list on st.
static int batch_launch(Batch& b, const BatchLaunch& L, cudaStream_t st) {
  {
    const int4* it = b.d_items + L.items_off;
    const unsigned n = (unsigned)L.nitems;
    if (L.kind == BK_FWD) {
      ProfScope ps(KIND_FWD, st);
      do {
        DDFAN_BATCH_ZL_NZ(8, 4, (go_fwd<8, 4>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 2, (go_fwd<8, 2>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 1, (go_fwd<8, 1>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 4, (go_fwd<4, 4>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 2, (go_fwd<4, 2>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 1, (go_fwd<4, 1>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 4, (go_fwd<2, 4>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 2, (go_fwd<2, 2>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 1, (go_fwd<2, 1>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 4, (go_fwd<1, 4>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 2, (go_fwd<1, 2>(b.d_fargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 1, (go_fwd<1, 1>(b.d_fargs, it, n, st)))
      } while (0);
    } else if (L.kind == BK_ADJ_X || L.kind == BK_ADJ_Y) {
      const bool xm = L.kind == BK_ADJ_X;
      ProfScope ps(xm ? KIND_BACK_A : KIND_BACK_B, st);
      do {
        DDFAN_BATCH_ZL_NZ(8, 4, (go_adj<8, 4>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 2, (go_adj<8, 2>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 1, (go_adj<8, 1>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 4, (go_adj<4, 4>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 2, (go_adj<4, 2>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 1, (go_adj<4, 1>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 4, (go_adj<2, 4>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 2, (go_adj<2, 2>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 1, (go_adj<2, 1>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 4, (go_adj<1, 4>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 2, (go_adj<1, 2>(xm, b.d_aargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 1, (go_adj<1, 1>(xm, b.d_aargs, it, n, st)))
      } while (0);
    } else {
      ProfScope ps(KIND_BACK_A, st);
      do {
        DDFAN_BATCH_ZL_NZ(8, 4, (go_ref<8, 4>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 2, (go_ref<8, 2>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(8, 1, (go_ref<8, 1>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 4, (go_ref<4, 4>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 2, (go_ref<4, 2>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(4, 1, (go_ref<4, 1>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 4, (go_ref<2, 4>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 2, (go_ref<2, 2>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(2, 1, (go_ref<2, 1>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 4, (go_ref<1, 4>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 2, (go_ref<1, 2>(b.d_rargs, it, n, st)))
        DDFAN_BATCH_ZL_NZ(1, 1, (go_ref<1, 1>(b.d_rargs, it, n, st)))
      } while (0);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batched launch (kind %d): %s", L.kind, cudaGetErrorString(e));
  }
  return DDFAN_OK;
}

// The launches of one batched iteration (every solve's next iteration).  With
// several solver groups each group's launches form a chain of their own on a
// side stream forked from st and joined back before FISTA (under capture:
// parallel branches of the graph), so one group's forward projections run
// beside another's backprojections, as separate solves on separate streams
// do; within a group the launches keep the step order.
static int batch_iteration(Batch& b, cudaStream_t st) {
  const bool fork = b.groups > 1 && !b.side.empty();
  cudaError_t e = cudaSuccess;
  if (fork) {
    e = cudaEventRecord(b.fork, st);
    for (size_t t = 0; t < b.side.size() && e == cudaSuccess; ++t) e = cudaStreamWaitEvent(b.side[t], b.fork, 0);
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch: fork: %s", cudaGetErrorString(e));
  }
  for (const BatchLaunch& L : b.launches) {
    const cudaStream_t q = fork && L.group > 0 ? b.side[L.group - 1] : st;
    const int rc = batch_launch(b, L, q);
    if (rc) return rc;
  }
  if (fork) {
    for (size_t t = 0; t < b.side.size() && e == cudaSuccess; ++t) {
      e = cudaEventRecord(b.join[t], b.side[t]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b.join[t], 0);
    }
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch: join: %s", cudaGetErrorString(e));
  }
  if (b.nfista) {
    ProfScope ps(KIND_FISTA, st);
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((b.fista_max + 255) / 256, 1024));
    k_fista_batch<<<dim3(blocks, b.nfista), 256, 0, st>>>(b.d_fista);
    k_fista_t_batch<<<(b.nfista + 127) / 128, 128, 0, st>>>(b.d_fista, b.nfista);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batched fista: %s", cudaGetErrorString(e));
  }
  return DDFAN_OK;
}

static int batch_create(Batch** out, Solver* const* solvers, int n) {
  *out = nullptr;
  if (!solvers || n < 1) return set_err(DDFAN_ERR_ARG, "batch: no solvers");
  std::unique_ptr<Batch, void (*)(Batch*)> B(new Batch(), batch_free);
  Batch& b = *B;
  for (int i = 0; i < n; ++i) {
    Solver* s = solvers[i];
    if (!s) return set_err(DDFAN_ERR_ARG, "batch: solver %d is null", i);
    if (!s->direct)
      return set_err(DDFAN_ERR_UNSUPPORTED,
                     "batch: solver %d is not a direct-mode solver with one angle list for all slices", i);
    if (i && s->device != solvers[0]->device)
      return set_err(DDFAN_ERR_ARG, "batch: solvers on devices %d and %d", solvers[0]->device, s->device);
    for (int j = 0; j < i; ++j)
      if (solvers[j] == s) return set_err(DDFAN_ERR_ARG, "batch: solver %d appears twice", i);
    b.sv.push_back(s);
  }
  b.device = solvers[0]->device;
  DeviceGuard g(b.device);
  {
    const int rc = batch_prepare_device(b.device);
    if (rc) return rc;
  }
  int maxsub = 0;
  for (Solver* s : b.sv) maxsub = std::max(maxsub, s->nsub);
  std::vector<DdFwdArgs> fargs;
  std::vector<DdAdjArgs> aargs;
  std::vector<DdRefArgs> rargs;
  std::vector<int4> items;
  // solver groups: largest solves first, dealt round robin
  int G = DDFAN_BATCH_GROUPS;
  if (const char* v = getenv("DDFAN_BATCH_GROUPS")) G = atoi(v);
  G = std::max(1, std::min(G, (int)b.sv.size()));
  b.groups = G;
  std::vector<int> group_of(b.sv.size());
  {
    std::vector<int> order(b.sv.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    auto work = [&](int i) { const Solver& s = *b.sv[i]; return (double)s.XN * s.YN * s.Zi * s.PNall; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) > work(y); });
    for (size_t r = 0; r < order.size(); ++r) group_of[order[r]] = (int)(r % G);
  }
  // per group, per step: class -> items, for each kind
  for (int grp = 0; grp < G; ++grp)
  for (int k = 0; k < maxsub; ++k) {
    std::map<std::pair<int, int>, std::vector<int4>> fwd, adjx, adjy, ref;
    for (size_t si = 0; si < b.sv.size(); ++si) {
      if (group_of[si] != grp) continue;
      Solver& s = *b.sv[si];
      if (k >= s.nsub) continue;
      const Plan& p = *s.P;
      const int o = s.off[k], c = s.cnt[k];
      if (c < 1) continue;
      const bool adj = s.back_mode == DDFAN_BACK_ADJ;
      const ViewGeom* vg = s.d_vg + o;
      const double2* fc = s.d_fc + (size_t)o * (s.U + 1);
      const float* cvd = s.d_cvd + (size_t)o * s.U;
      DdResidual r;
      r.y = s.d_y; r.yview = s.d_yview + o; r.rowsum = s.d_rows + (size_t)o * s.U; r.wgt = adj ? cvd : nullptr;
      r.ystride = s.Zi;
      const DdFwdArgs fa = make_fwd_dd_args(p, s.d_x, vg, fc, cvd, s.d_order + o, c, s.d_ax, s.U + 1, s.Zi, 0, s.Zi, &r);
      if (fa.nzt < 1) continue;
      const int fnz = dd_nz(fa.nzt, fa.nzc);
      const int fi = (int)fargs.size();
      fargs.push_back(fa);
      const int cw = fwd_cw(p.ZL, fnz), ncb = (s.U + cw - 1) / cw, nzg = (fa.nzt + fnz - 1) / fnz;
      // z-tile groups outermost and the rest in the single-solve grid's
      // order: the CTAs in flight share one group's slices, whose image part
      // then stays in L2
      auto& fl = fwd[{p.ZL, fnz}];
      for (int zg = 0; zg < nzg; ++zg) {
        if (DDFAN_DD_FWD_ROWS_X) {
          for (int cb = 0; cb < ncb; ++cb)
            for (int row = 0; row < c; ++row) fl.push_back(make_int4(fi, row, cb, zg));
        } else {
          for (int row = 0; row < c; ++row)
            for (int cb = 0; cb < ncb; ++cb) fl.push_back(make_int4(fi, row, cb, zg));
        }
      }
      BackEpi e{};
      e.out = s.d_x; e.xin = s.d_x; e.colsum = s.d_cols + (size_t)k * s.XN * s.YN;
      e.nonneg = s.nonneg; e.mask = p.has_mask ? p.d_mask : nullptr; e.zlo = 0; e.zhi = s.Zi;
      int rc = check_back_dd(p, s.back_mode, s.d_order + o, s.d_counts + 2 * k);
      if (rc) return rc;
      DdAdjArgs a1, a2;
      DdRefArgs ar;
      const int nzt = make_back_dd_args(p, s.back_mode, s.d_ax, vg, fc, s.d_order + o, s.d_counts + 2 * k, c, e, &a1,
                                        &a2, &ar);
      if (adj) {
        const int bnz = dd_nz(nzt, p.NZ), nbz = (nzt + bnz - 1) / bnz;
        int LT, KT;
        adj_tile(p.ZL, &LT, &KT);
        const int i1 = (int)aargs.size();
        aargs.push_back(a1);
        aargs.push_back(a2);
        const int tx = ((s.XN + LT - 1) / LT) * ((s.YN + KT - 1) / KT);  // x columns as lines
        const int ty = ((s.YN + LT - 1) / LT) * ((s.XN + KT - 1) / KT);  // y rows as lines
        auto& lx = adjx[{p.ZL, bnz}];
        auto& ly = adjy[{p.ZL, bnz}];
        for (int zg = 0; zg < nbz; ++zg)
          for (int t = 0; t < tx; ++t) lx.push_back(make_int4(i1, t, zg, 0));
        for (int zg = 0; zg < nbz; ++zg)
          for (int t = 0; t < ty; ++t) ly.push_back(make_int4(i1 + 1, t, zg, 0));
      } else {
        const int bnz = dd_nz(nzt, p.NZ), nbz = (nzt + bnz - 1) / bnz;
        int LT, KT;
        adj_tile(p.ZL, &LT, &KT);  // the REF kernel uses the exact adjoint's voxel tile
        const int ri = (int)rargs.size();
        rargs.push_back(ar);
        const int tiles = ((s.YN + LT - 1) / LT) * ((s.XN + KT - 1) / KT);
        auto& lr = ref[{p.ZL, bnz}];
        for (int zg = 0; zg < nbz; ++zg)
          for (int t = 0; t < tiles; ++t) lr.push_back(make_int4(ri, t, zg, 0));
      }
    }
    auto emit = [&](int kind, std::map<std::pair<int, int>, std::vector<int4>>& m) {
      for (auto& kv : m) {
        if (kv.second.empty()) continue;
        BatchLaunch L{kind, kv.first.first, kv.first.second, items.size(), kv.second.size(), grp};
        items.insert(items.end(), kv.second.begin(), kv.second.end());
        b.launches.push_back(L);
      }
    };
    emit(BK_FWD, fwd);
    emit(BK_ADJ_X, adjx);
    emit(BK_REF, ref);
    emit(BK_ADJ_Y, adjy);
  }
  for (const BatchLaunch& L : b.launches)
    if (L.nitems > (size_t)INT_MAX) return set_err(DDFAN_ERR_UNSUPPORTED, "batch: %zu CTAs in one launch", L.nitems);
  std::vector<FistaDesc> fista;
  for (Solver* s : b.sv)
    if (s->useFISTA) {
      const size_t V = (size_t)s->XN * s->YN * s->Zi;
      fista.push_back(FistaDesc{s->d_x, s->d_xprev, V, s->d_t});
      b.fista_max = std::max(b.fista_max, V);
    }
  b.nfista = (int)fista.size();
  b.kernel_launches = (int)b.launches.size() + (b.nfista ? 2 : 0);
  cudaError_t e = cudaStreamCreateWithFlags(&b.own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b.last_use, cudaEventDisableTiming);
  if (b.groups > 1) {
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming);
    for (int t = 1; t < b.groups && e == cudaSuccess; ++t) {
      cudaStream_t q = nullptr;
      cudaEvent_t ev = nullptr;
      e = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking);
      if (e == cudaSuccess) b.side.push_back(q);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) b.join.push_back(ev);
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(DDFAN_ERR_CUDA, "batch: stream/event creation: %s", cudaGetErrorString(e));
  }
  int rc;
  auto up = [&](auto** dst, auto& vec) -> int {
    if (vec.empty()) return DDFAN_OK;
    const size_t bytes = sizeof(vec[0]) * vec.size();
    int r = dev_alloc((void**)dst, bytes, b.own);
    if (r) return r;
    cudaError_t ee = cudaMemcpyAsync(*dst, vec.data(), bytes, cudaMemcpyHostToDevice, b.own);
    if (ee != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch: upload: %s", cudaGetErrorString(ee));
    return DDFAN_OK;
  };
  if ((rc = up(&b.d_fargs, fargs)) || (rc = up(&b.d_aargs, aargs)) || (rc = up(&b.d_rargs, rargs)) ||
      (rc = up(&b.d_items, items)) || (rc = up(&b.d_fista, fista)))
    return rc;
  // the pageable sources above are consumed before they go out of scope
  e = cudaStreamSynchronize(b.own);
  if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch: upload: %s", cudaGetErrorString(e));
  *out = B.release();
  return DDFAN_OK;
}

}  // namespace ddfan

using namespace ddfan;

extern "C" {

DDFAN_API int ddfan_batch_create(ddfan_batch** out, ddfan_ossart* const* solvers, int n) {
  if (!out) return set_err(DDFAN_ERR_ARG, "out is null");
  Batch* b = nullptr;
  int rc = batch_create(&b, reinterpret_cast<Solver* const*>(solvers), n);
  *out = reinterpret_cast<ddfan_batch*>(b);
  return rc;
}

DDFAN_API void ddfan_batch_destroy(ddfan_batch* b) { batch_free(reinterpret_cast<Batch*>(b)); }

DDFAN_API int ddfan_batch_launches_per_iter(const ddfan_batch* h) {
  const Batch* b = reinterpret_cast<const Batch*>(h);
  return b ? b->kernel_launches : 0;
}

DDFAN_API int ddfan_batch_iterate(ddfan_batch* h, int numOfIter, int use_graph, void* stream) {
  Batch* b = reinterpret_cast<Batch*>(h);
  if (!b || numOfIter < 0) return set_err(DDFAN_ERR_ARG, "batch_iterate: bad argument");
  DeviceGuard g(b->device);
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (!use_graph) {
    for (int it = 0; it < numOfIter; ++it)
      if ((rc = batch_iteration(*b, st))) return rc;
  } else {
    if (!b->gexec) {
      cudaError_t e = cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e));
      rc = batch_iteration(*b, b->own);
      cudaGraph_t gr = nullptr;
      e = cudaStreamEndCapture(b->own, &gr);
      if (rc) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e));
      b->graph = gr;
      e = cudaGraphInstantiate(&b->gexec, b->graph, 0);
      if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch graph: %s", cudaGetErrorString(e));
    }
    for (int it = 0; it < numOfIter; ++it) {
      cudaError_t e = cudaGraphLaunch(b->gexec, st);
      if (e != cudaSuccess) return set_err(DDFAN_ERR_CUDA, "batch graph launch: %s", cudaGetErrorString(e));
    }
  }
  for (Solver* s : b->sv)
    if ((rc = solver_after_iterations(*s, numOfIter, st))) return rc;
  cudaEventRecord(b->last_use, st);
  return DDFAN_OK;
}

}  // extern "C"
