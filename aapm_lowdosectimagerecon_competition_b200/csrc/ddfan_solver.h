// ddfan_solver.h -- the OS-SART solver's state, shared by the solver
// (ddfan_solver.cu) and the batched launches over many solvers (ddfan_batch.cu).
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "ddfan.h"
#include "ddfan_device.cuh"
#include "ddfan_plan.h"

namespace ddfan {

struct Solver {
  Plan* P = nullptr;  // Zi slices, PNmax = largest subset (or largest tile view range)
  int device = 0;
  int PNall = 0, nsub = 1, useFISTA = 1, nonneg = 0, back_mode = DDFAN_BACK_REF;
  int XN = 0, YN = 0, U = 0, Z = 0;
  std::vector<int> off, cnt;  // subset k: rows [off[k], off[k] + cnt[k]) of the subset-ordered tables
  ViewGeom* d_vg = nullptr;
  double2* d_fc = nullptr;
  float* d_cvd = nullptr;
  int* d_yview = nullptr;  // subset-ordered row -> original view index
  int* d_order = nullptr;  // per subset (or per subset and z-tile): views in dispatch order (x-major first)
  int* d_counts = nullptr; // per subset: {x-major views, others}
  float* d_rows = nullptr; // [PNall][U]   row sums, subset order
  float* d_cols = nullptr; // [nsub][YN][XN] column sums
  float* d_y = nullptr;    // [PNall][U][Zi] measured sinogram
  float* d_x = nullptr;    // [YN][XN][Zi] image
  float* d_xprev = nullptr;
  float* d_ax = nullptr;   // [PNmax][U][Zi]
  double* d_t = nullptr;
  // Per-slice view angles ("windowed" solver).  Every slice's list is a
  // window of one table of raw views (view ib of slice z is raw view
  // off_z + ib): the geometry rows are raw views, grouped by raw view mod
  // numOfOS (row = (g mod nOS) * Mc + g / nOS).  Internally slices are
  // reordered so that a z-tile holds slices of one residue off_z mod nOS --
  // they then need the same raw views for each subset -- and each class is
  // padded to whole z-tiles; z-tile zt of subset k projects the raw views of
  // its residue class that fall in its slices' windows.
  bool win = false;
  int Zi = 0;                // internal slices (Z when not windowed)
  int nzt = 0, Mc = 1;
  std::vector<int> perm;     // internal slice -> original slice, -1 for padding
  int* d_perm = nullptr;     // the same on the device
  int* d_inv = nullptr;      // original slice -> internal slice
  int* d_soff = nullptr;     // internal slice -> window offset (INT_MAX for padding)
  int4* d_ztd = nullptr;     // [nsub][nzt] view ranges
  std::vector<int> maxcnt;   // per subset: largest range of a z-tile
  float* d_xu = nullptr;     // [YN][XN][Z] image in the caller's layout
  float* d_stage = nullptr;  // [PNall][U][Z] host sinogram staging (windowed, slice-major)
  // Per-slice view angles, slice-major path: every slice keeps its own
  // geometry (rows z * cstride + m: view k + m * numOfOS of slice z in
  // subset k, rebuilt per subset) and the image, sinogram and prefix-sum
  // tables are slice-major: d_x [Z][YN][XN], d_y [Z][PNall][U],
  // d_ax [Z][cstride][U].
  bool ps = false;
  int cstride = 0;
  float* d_pang = nullptr;   // [nsub][Z][cstride] angles of each slice's views per subset
  float* d_xt = nullptr;     // [Z][XN][YN] image columns
  float* d_tabx = nullptr;   // image rows table [Z][YN][XN] cells
  float* d_taby = nullptr;   // image columns table [Z][XN][YN] cells
  float* d_sq = nullptr;     // weighted residual table [Z][cstride][U+1] cells
  // Direct mode (no prefix-sum tables; one angle list for all slices): the
  // image d_x [YN][XN][Zi] has its slices padded to a multiple of 4 (Zi) and
  // its masked voxels kept at 0, so the projector reads it as it is; d_ax holds
  // the residual [PNmax][U+1][Zi] with a zero guard channel.  A masked voxel's
  // published value is its initial one (d_x0, the caller's layout), clamped
  // at 0 by the updates when they clamp -- what the table path computes there.
  bool direct = false;
  float* d_x0 = nullptr;
  long long iters_done = 0;
  cudaStream_t own = nullptr;
  cudaEvent_t last_use = nullptr;  // recorded after work enqueued on a caller's stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  size_t bytes = 0;
  int launches = 0;
};

// After n iterations enqueued on st outside ddfan_ossart_iterate: count them
// and publish the image callers read (masked / padded / reordered layouts).
int solver_after_iterations(Solver& s, int n, cudaStream_t st);

}  // namespace ddfan
