/*
 * ddfan.h -- C ABI of the B200 fan-beam multi-slice distance-driven (DD)
 * projector / backprojector and OS-SART solver (libddfan.so).
 *
 * Every entry point returns a status code (DDFAN_OK on success) and never
 * exits the process; ddfan_last_error() gives a message for the calling
 * thread's last failure.  No entry point resets a device.
 *
 * Array layouts are the C (row-major) views of the reference's MATLAB arrays,
 * so buffers pass through unchanged:
 *   image    vol [YN][XN][SLN]   float   (MATLAB single(SLN, XN, YN))
 *   sinogram prj [PN][DNU][SLN]  float   (MATLAB single(SLN, DNU, PN))
 *   angles   hangs[PN][SLN]      float   (MATLAB single(SLN, PN)), radians
 *   mask     mask [YN][XN]       uint8   (first XN*YN bytes of MATLAB [mask, mask'])
 * Reference paths below are relative to the reference project root.
 */
#ifndef DDFAN_H
#define DDFAN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DDFAN_API __attribute__((visibility("default")))
#else
#define DDFAN_API
#endif

/* status codes */
#define DDFAN_OK 0
#define DDFAN_ERR_ARG 1         /* invalid argument (sizes, null pointers, modes) */
#define DDFAN_ERR_CUDA 2        /* a CUDA runtime call failed */
#define DDFAN_ERR_NOMEM 3       /* device or host allocation failed / over budget */
#define DDFAN_ERR_UNSUPPORTED 4 /* geometry or size outside what the kernels handle */
#define DDFAN_ERR_BUSY 5        /* resource in use (serving slots) */

/* precision of the prefix-sum (SAT) tables and of their differences */
#define DDFAN_SAT_FP32 0 /* plain FP32 sums (the reference's precision class) */
#define DDFAN_SAT_HILO 1 /* compensated hi/lo FP32 pairs */
#define DDFAN_SAT_FP64 2 /* FP64 sums */
/* no tables: each difference of two interpolated prefix sums is evaluated as
 * the sum of the values it telescopes to (exact overlap weights, FP32, no
 * cancellation).  Used on the paths with one angle list for all slices; paths
 * that keep tables (per-slice angle lists) use hi/lo cells in this mode. */
#define DDFAN_SAT_DIRECT 3

/* backprojector */
#define DDFAN_BACK_REF 0 /* the reference backprojector's formula (MultiSlicesBackGPU.cu:115-184) */
#define DDFAN_BACK_ADJ 1 /* exact transpose of the forward projector */

DDFAN_API const char* ddfan_last_error(void);
DDFAN_API int ddfan_version(void);

/* ---- tile selection and memory estimates (serving / autotuning) ----
 * No counterpart in the reference.  Plans split the slices into z-tiles of
 * zl 4-slice blocks (zl in {1, 2, 4, 8}); by default a cost model picks zl
 * for a stack of `zblocks` blocks, ddfan_tune_set_zl records a measured
 * choice (zl = 0 forgets it).  Process-wide, thread-safe; affects plans
 * created afterwards. */
DDFAN_API int ddfan_tune_set_zl(int zblocks, int zl);
DDFAN_API int ddfan_tune_get_zl(int zblocks);
/* the direct mode's (DDFAN_SAT_DIRECT) second tile dimension: each thread
 * walks the footprints it decodes for up to nz z-tiles (nz in {1, 2, 4};
 * default 4; nz = 0 forgets a record).  Results do not depend on it (every
 * slice sums the same terms in the same order); the launch shape does. */
DDFAN_API int ddfan_tune_set_nz(int zblocks, int nz);
DDFAN_API int ddfan_tune_get_nz(int zblocks);
/* device bytes ddfan_plan_create / ddfan_ossart_create would allocate
 * (the solver figure includes its transient set-up buffers); 0 = bad sizes.
 * Both are for one angle list shared by all slices.  Per-slice lists take
 * more: a solver on the slice-major path about 16 B x (XN+2) x (YN+2) x SLN
 * x 2 for its tables plus 2 x 4 B x PNall x DNU x SLN for the sinogram and
 * its staging, and a plan's first per-slice call on the slice-major kernels
 * about 40 B x (DNU+1) x PNmax x SLN plus the same image tables. */
DDFAN_API size_t ddfan_plan_estimate_bytes(int XN, int YN, int DNU, int SLN, int PNmax, int sat_mode);
DDFAN_API size_t ddfan_ossart_estimate_bytes(int XN, int YN, int DNU, int SLN, int PNall, int numOfOS,
                                             int sat_mode);

/* Source position and channel centres on the arc detector, as the MATLAB
 * wrapper builds them (replaces AAPM_script/DD2MutiSlices.m:49-76):
 * stepTheta = 2 atan(detCellWidth / 2 / sdd), beta_i = (i - detCntIdx) stepTheta
 * for 1-based i, xds_i = sdd sin(beta_i), yds_i = sid - sdd cos(beta_i),
 * source (x0, y0) = (0, sid).  Single-precision arithmetic like MATLAB's. */
DDFAN_API int ddfan_fan_geometry(float sid, float sdd, int DNU, float detCellWidth, float detCntIdx,
                                 float* x0, float* y0, float* xds, float* yds);

/* ---- mex-compatible host entry points (host pointers, synchronous) ----
 * Replaces the MEX function MultiSlicesProjGPU
 * (AAPM_script/MultiSlicesProjGPU.cu:550-575 -> DD2ProjMultiGPUs_CPP17 :486-547):
 * the same 16 inputs in the same order, then the SAT precision and the output
 * buffer prj[PN][DNU][SLN] (the mex allocates it; here the caller does).
 * startIdx[nStartIdx] gives the first slice of each device's slab
 * (DD2MutiSlices.m:95-101); slab k runs on device k mod (device count), each
 * device's slabs on a host thread of its own so that devices work at the same
 * time (as the reference's one std::thread per GPU, MultiSlicesProjGPU.cu:
 * 474-484); nStartIdx <= 0 or startIdx == NULL means one slab on the current
 * device. */
DDFAN_API int ddfan_MultiSlicesProjGPU(float x0, float y0, int DNU, const float* xds,
                                       const float* yds, float imgXCenter, float imgYCenter,
                                       const float* hangs, int PN, int XN, int YN, int SLN,
                                       const float* vol, float dx, const uint8_t* mask,
                                       const int32_t* startIdx, int nStartIdx, int sat_mode,
                                       float* prj);

/* Replaces the MEX function MultiSlicesBackGPU
 * (AAPM_script/MultiSlicesBackGPU.cu:409-436 -> DD2BackMultiGPUs :349-406):
 * the same 17 inputs in the same order, then SAT precision, backprojector
 * (DDFAN_BACK_REF reproduces the reference; DDFAN_BACK_ADJ is the exact
 * transpose of ddfan_MultiSlicesProjGPU) and the output vol[YN][XN][SLN].
 * Voxels whose mask byte is 0 are written as 0. */
DDFAN_API int ddfan_MultiSlicesBackGPU(float x0, float y0, int DNU, const float* xds,
                                       const float* yds, float detCntIdx, float imgXCenter,
                                       float imgYCenter, const float* hangs, int PN, int XN,
                                       int YN, int SLN, const float* prj, float dx,
                                       const uint8_t* mask, const int32_t* startIdx,
                                       int nStartIdx, int sat_mode, int back_mode, float* vol);

/* ---- device API: a plan owns the geometry and the scratch tables ----
 * Replaces the per-call set-up of DD2::DD2_gpu_proj_branchless_sat2d
 * (AAPM_script/MultiSlicesProjGPU.cu:211-385) and DD2_gpu_back
 * (AAPM_script/MultiSlicesBackGPU.cu:187-268): boundaries, image-centre
 * index, mask upload and table allocation happen once, not per call. */
typedef struct ddfan_plan_s ddfan_plan;

DDFAN_API int ddfan_plan_create(ddfan_plan** out, float x0, float y0, int DNU, const float* xds,
                                const float* yds, float detCntIdx, float imgXCenter,
                                float imgYCenter, int XN, int YN, float dx,
                                const uint8_t* mask /* host [YN][XN], NULL = all ones */,
                                int SLN, int PNmax, int sat_mode, int device);
DDFAN_API void ddfan_plan_destroy(ddfan_plan* plan);
/* device bytes held by the plan */
DDFAN_API size_t ddfan_plan_device_bytes(const ddfan_plan* plan);

/* Plans, solvers and rebinning calls take device memory, stream-ordered,
 * from one pool per device that the library owns; memory they free stays
 * in that pool for the next ones (no new mapping per solve).  Bytes the
 * pool holds unused, and a call that returns them to the driver (it
 * synchronises the device first).  No reference counterpart: the mex
 * functions allocate and free on every call. */
DDFAN_API size_t ddfan_cached_bytes(int device);
DDFAN_API int ddfan_release_cached(int device);

/* Forward projection of device vol[YN][XN][SLN] into device prj[PN][DNU][SLN].
 * d_angs: device view angles; angs_per_slice = 0: d_angs[PN] shared by all
 * slices; 1: d_angs[PN][SLN] (the reference's hangs layout; slices with the
 * same list are projected together, and when many lists differ -- rebinned
 * data -- every slice runs with its own geometry on slice-major kernels,
 * whose buffers the plan allocates on the first such call).  Asynchronous on
 * `stream` (a cudaStream_t, NULL = legacy default stream). */
DDFAN_API int ddfan_proj_dev(ddfan_plan* plan, const float* d_angs, int PN, int angs_per_slice,
                             const float* d_vol, float* d_prj, void* stream);
/* Backprojection of device prj[PN][DNU][SLN] into device vol[YN][XN][SLN]. */
DDFAN_API int ddfan_back_dev(ddfan_plan* plan, const float* d_angs, int PN, int angs_per_slice,
                             const float* d_prj, float* d_vol, int back_mode, void* stream);

/* Forward projection that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc: their device memory is
 * owned up front by another allocator (a framework's caching allocator, a pool
 * reserved at start-up), or they cannot take cudaMalloc's implicit device-wide
 * synchronisation mid-pipeline.  Same result as ddfan_proj_dev on a plan of the
 * same geometry and sat_mode (any of the four); device inputs d_angs[PN] (one
 * angle list for all slices) and d_vol[YN][XN][SLN], device output
 * d_prj[PN][DNU][SLN]; xds, yds and mask (may be NULL) are host arrays, read
 * before the call returns.  Runs on the calling thread's current device.
 * All scratch (geometry and prefix-sum tables, or the staged image of the
 * direct mode) lives in one fixed device array of DDFAN_NOALLOC_SCRATCH_BYTES
 * that every GPU loading this library holds until exit; a problem needing more
 * returns DDFAN_ERR_UNSUPPORTED before any GPU work.  The first call on a device
 * -- and the first after a cudaDeviceReset, which gives the device a new
 * context -- looks up that array's device address (cudaGetSymbolAddress) and
 * allows the direct-mode forward kernels their shared memory
 * (cudaFuncSetAttribute); make that first call before any stream capture.  A call made while its
 * stream is being captured returns DDFAN_ERR_UNSUPPORTED: every call uploads
 * its geometry from host memory that is gone when it returns.  Calls share
 * the array, so calls whose kernels overlap on one GPU race: serialise them
 * (one stream, or events). */
#define DDFAN_NOALLOC_SCRATCH_BYTES (64ull << 20)
DDFAN_API int ddfan_proj_noalloc(float x0, float y0, int DNU, const float* xds, const float* yds,
                                 float imgXCenter, float imgYCenter, const float* d_angs, int PN,
                                 int XN, int YN, int SLN, const float* d_vol, float dx,
                                 const uint8_t* mask, int sat_mode, float* d_prj, void* stream);

/* ---- OS-SART / FISTA solver with device-resident state ----
 * Replaces AAPM_script/OSSART_AAPM.m:33-118.  Subset k holds views
 * k, k + numOfOS, ... (:60); row/column sums come from slice 0 (:61-64);
 * where a sum is 0 the value is left un-normalised (:88, :94); FISTA momentum
 * after each iteration (:111-115).  nonneg != 0 clamps the image at 0 after
 * every subset update (an addition).  Each iteration is one CUDA graph. */
typedef struct ddfan_ossart_s ddfan_ossart;

DDFAN_API int ddfan_ossart_create(ddfan_ossart** out, float x0, float y0, int DNU,
                                  const float* xds, const float* yds, float detCntIdx,
                                  float imgXCenter, float imgYCenter, const float* hangs,
                                  int PNall, int XN, int YN, int SLN, float dx,
                                  const uint8_t* mask, int numOfOS, int useFISTA, int nonneg,
                                  int sat_mode, int back_mode, int device);
DDFAN_API void ddfan_ossart_destroy(ddfan_ossart* s);
DDFAN_API size_t ddfan_ossart_device_bytes(const ddfan_ossart* s);
/* measured sinogram proj[PNall][DNU][SLN]: host (to_device = 0 -> copied in
 * with cudaMemcpyAsync) or device pointer (is_device = 1 -> copied D2D). */
DDFAN_API int ddfan_ossart_set_sinogram(ddfan_ossart* s, const float* proj, int is_device,
                                        void* stream);
/* initial image [YN][XN][SLN], host or device; resets the FISTA state. */
DDFAN_API int ddfan_ossart_set_image(ddfan_ossart* s, const float* img, int is_device,
                                     void* stream);
/* run numOfIter iterations on `stream` (graph per iteration when use_graph != 0) */
DDFAN_API int ddfan_ossart_iterate(ddfan_ossart* s, int numOfIter, int use_graph, void* stream);
/* copy the current image out (host or device destination) */
DDFAN_API int ddfan_ossart_get_image(ddfan_ossart* s, float* img, int is_device, void* stream);
/* device pointer of the current image (valid until the solver is destroyed) */
DDFAN_API float* ddfan_ossart_image_ptr(ddfan_ossart* s);
/* Runs numOfIter iterations without a graph, each kernel launch bracketed by
 * CUDA events on `stream`; returns per kind the summed device milliseconds
 * and launch counts.  Kinds: 0 view geometry, 1 image prefix sums,
 * 2 forward projection, 3 sinogram prefix sums (+ residual), 4 backprojection
 * (REF, or exact-adjoint column pass), 5 exact-adjoint row pass, 6 FISTA.
 * Arrays must hold 7 entries.  (Diagnostics; no counterpart in the reference.) */
DDFAN_API int ddfan_ossart_profile(ddfan_ossart* s, int numOfIter, void* stream, float* ms_by_kind,
                                   int* launches_by_kind);
/* number of kernel launches one iteration issues */
DDFAN_API int ddfan_ossart_launches_per_iter(const ddfan_ossart* s);

/* ---- batched OS-SART: many reconstructions advanced together ----
 * No counterpart in the reference, which runs one reconstruction per MATLAB
 * call (AAPM_script/OSSART_AAPM.m:85, :92).  Groups n solvers created with
 * DDFAN_SAT_DIRECT and one angle list for all slices (any sizes, subset
 * counts, backprojectors; one device).  Each ddfan_batch_iterate iteration
 * runs every solver's next OS-SART iteration with one launch per kernel
 * kind, subset step and tile class over a device work list of all solvers'
 * work items (view x channel block x slice tiles; voxel tiles x slice tiles),
 * captured as one CUDA graph when use_graph != 0; each solver computes
 * exactly what ddfan_ossart_iterate computes for it alone.  The batch does
 * not own the solvers: they must outlive it, and their sinograms and images
 * must be set (ordered before the iterate call's stream) first.  Results are
 * read with ddfan_ossart_get_image. */
typedef struct ddfan_batch_s ddfan_batch;

DDFAN_API int ddfan_batch_create(ddfan_batch** out, ddfan_ossart* const* solvers, int n);
DDFAN_API void ddfan_batch_destroy(ddfan_batch* b);
DDFAN_API int ddfan_batch_iterate(ddfan_batch* b, int numOfIter, int use_graph, void* stream);
/* kernel launches one batched iteration issues */
DDFAN_API int ddfan_batch_launches_per_iter(const ddfan_batch* b);

/* One-call host entry mirroring OSSART_AAPM(Proj, Views, initImg, conf,
 * numOfIter, numOfOS, mask, useFISTA) with the geometry already expanded. */
DDFAN_API int ddfan_OSSART_AAPM(float x0, float y0, int DNU, const float* xds, const float* yds,
                                float detCntIdx, float imgXCenter, float imgYCenter,
                                const float* proj, const float* hangs, int PNall, int XN, int YN,
                                int SLN, float dx, const float* initImg, const uint8_t* mask,
                                int numOfIter, int numOfOS, int useFISTA, int nonneg,
                                int sat_mode, int back_mode, float* reconImg);

/* ---- Helical-to-fan single-slice rebinning ----
 * Replaces the CPU mex HelicalToFan (AAPM_script/HelicalToFanFunc_mex.cpp:142-185,
 * per-slice body HelicalToFanImpl :41-139; MATLAB entry HelicalToFanFunc_mex
 * called from HelicalToFan_routine.m:39-42) with the same argument meaning and a
 * bit-identical result.  proj: raw helical views [nViews][DetWidth][DetHeight]
 * (MATLAB (Height, Channel, View)); zPos[SLN] target slice positions; outputs in
 * the mex's layouts Proj[SLN][DefTimes][DetWidth] and Views[SLN][DefTimes].
 * nViews is the number of raw views (the mex reads it from the array; a slice
 * that needs a view beyond it is DDFAN_ERR_ARG, where the reference reads past
 * its buffer).  A slice with floor((z - h/2) / deltaZ) < 0 is all zero, as in
 * the reference.  Host pointers; runs on the current device. */
DDFAN_API int ddfan_HelicalToFan(float* Proj, float* Views, const float* proj, long long nViews,
                                 const float* zPos, int SLN, float SD, float SO, float BVAngle,
                                 int DetWidth, int DetHeight, float PerDetW, float PerDetH,
                                 int DefTimes, float DetCenterW, float SpiralPitchFactor);
/* Device-resident variant: d_proj[nViews][DetWidth][DetHeight] on the device,
 * zPos on the host.  layout 0 writes the mex layouts above; layout 1 writes the
 * layouts HelicalToFan_routine.m:44-45 returns after its permutes,
 * d_Proj[DefTimes][DetWidth][SLN] and d_Views[DefTimes][SLN] (the sinogram
 * layout ddfan_ossart_set_sinogram takes).  Stream-ordered; no host sync. */
DDFAN_API int ddfan_helical_to_fan_dev(const float* d_proj, long long nViews, const float* zPos,
                                       int SLN, float SD, float SO, float BVAngle, int DetWidth,
                                       int DetHeight, float PerDetW, float PerDetH, int DefTimes,
                                       float DetCenterW, float SpiralPitchFactor, int layout,
                                       float* d_Proj, float* d_Views, void* stream);

/* DICOM-CT-PD projections on the device: the stored 16-bit pixels of nViews
 * projection files, d_pix[nViews][W][H] (DICOM rows = detector columns W,
 * DICOM columns = detector rows H), to the float raw views
 * d_proj[nViews][W][H] that ddfan_helical_to_fan_dev reads, view order
 * reversed when reverse != 0.  Replaces the conversion half of
 * AAPM_script/readProj.m:43-54 (double(dicomread(...)), permute, flip); the
 * files themselves are parsed on the host.  Buffers 16-byte aligned when
 * W * H is a multiple of 8.  Stream-ordered. */
DDFAN_API int ddfan_ctpd_views_to_raw(const uint16_t* d_pix, long long nViews, int W, int H, int reverse,
                                      float* d_proj, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DDFAN_H */
