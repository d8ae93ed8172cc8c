/*
 * ddfan_oracle.c -- FP64 CPU restatement of the reference's fan-beam
 * multi-slice distance-driven (DD) path.  TEST INFRASTRUCTURE ONLY: it is the
 * checker that tests/, smoke() and bench.py's CPU-baseline leg call; no
 * product code path links or calls it.
 *
 * What it restates (reference paths relative to the reference project root):
 *   boundaries       AAPM_script/utilities.cuh:268-287        (DD3Boundaries)
 *   angle wrap       AAPM_script/utilities.cuh:143-148        (regularizeAngle)
 *   cos/sin table    AAPM_script/utilities.cuh:218-227        (Constant_MultiSlice_host)
 *   image masking    AAPM_script/MultiSlicesProjGPU.cu:202-209 (maskingData)
 *   image SATs       AAPM_script/MultiSlicesProjGPU.cu:25-97   (zero-padded prefix sums)
 *   forward kernel   AAPM_script/MultiSlicesProjGPU.cu:100-200 + host :211-234
 *   sinogram SAT     AAPM_script/MultiSlicesBackGPU.cu:12-66
 *   back kernel      AAPM_script/MultiSlicesBackGPU.cu:115-184 + host :187-242 ("REF")
 *   OS-SART + FISTA  AAPM_script/OSSART_AAPM.m:49-118
 * plus the exact transpose of the forward ("ADJ"), which the reference does
 * not have.
 *
 * Semantics chosen where the reference is lossy or racy:
 *  - every quantity is carried in double; the only float roundings kept are
 *    the ones the reference's host code stores (input arrays, and the
 *    boundary arrays that DD3Boundaries<float> writes back as float);
 *  - texture fetches (cudaFilterModeLinear + cudaAddressModeClamp, unnormalised
 *    coordinates) are evaluated with exact weights: coordinate t samples the
 *    padded table at texel position clamp(t - 0.5, 0, W - 1), linearly
 *    interpolated -- the hardware's 8-bit weight fraction is not modelled;
 *  - the multi-GPU split/gather is the intended one (no skipped elements);
 *  - voxels whose mask byte is 0 are 0 in the back projections (the reference
 *    leaves them uninitialised).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_TWOPI 6.283185307179586 /* utilities.cuh:43 */

typedef struct {
  double x0, y0;        /* source position at view angle 0 */
  int DNU;              /* detector channels */
  const float* xds;     /* channel centres, DNU */
  const float* yds;
  double* bx;           /* boundaries, DNU + 1 (float-rounded like DD3Boundaries<float>) */
  double* by;
  double ocx, ocy;      /* image centre index (MultiSlicesProjGPU.cu:225-226) */
  double dx;            /* pixel size */
  int XN, YN;
  const uint8_t* mask;  /* [YN][XN] bytes, may be NULL (all ones) */
} geom_t;

/* utilities.cuh:143-148 */
static double wrap_angle(double c) {
  while (c >= ORC_TWOPI) c -= ORC_TWOPI;
  while (c < 0) c += ORC_TWOPI;
  return c;
}

/* utilities.cuh:268-287: boundaries from centres; the reference evaluates in
 * double (1.5 * float) and stores into a float array. */
void orc_boundaries(int ncenters, const float* c, double* out) {
  const int n = ncenters + 1;
  if (n >= 3) {
    for (int i = 0; i < n; ++i) {
      double v;
      if (i == 0) v = 1.5 * c[0] - 0.5 * c[1];
      else if (i == n - 1) v = 1.5 * c[i - 1] - 0.5 * c[i - 2];
      else v = 0.5 * c[i - 1] + 0.5 * c[i];
      out[i] = (double)(float)v;
    }
  } else {
    out[0] = (double)(float)(c[0] - 0.5);
    out[1] = (double)(float)(c[0] + 0.5);
  }
}

static int geom_init(geom_t* g, float x0, float y0, int DNU, const float* xds, const float* yds,
                     float imgXCenter, float imgYCenter, int XN, int YN, float dx,
                     const uint8_t* mask) {
  g->x0 = x0; g->y0 = y0; g->DNU = DNU; g->xds = xds; g->yds = yds;
  g->dx = dx; g->XN = XN; g->YN = YN; g->mask = mask;
  g->ocx = (XN - 1.0) * 0.5 - (double)imgXCenter / (double)dx;
  g->ocy = (YN - 1.0) * 0.5 - (double)imgYCenter / (double)dx;
  g->bx = (double*)malloc(sizeof(double) * (DNU + 1));
  g->by = (double*)malloc(sizeof(double) * (DNU + 1));
  if (!g->bx || !g->by) return -1;
  orc_boundaries(DNU, xds, g->bx);
  orc_boundaries(DNU, yds, g->by);
  return 0;
}

static void geom_free(geom_t* g) { free(g->bx); free(g->by); }

/* Linear interpolation of a zero-padded prefix-sum table of W entries at
 * texel coordinate t (texture semantics: sample position t - 0.5, clamped). */
static inline double sat_fetch(const double* S, int W, double t) {
  double c = t - 0.5;
  if (!(c > 0.0)) c = 0.0;
  if (c > (double)(W - 1)) c = (double)(W - 1);
  int i = (int)floor(c);
  if (i >= W - 1) return S[W - 1];
  double f = c - (double)i;
  return S[i] + f * (S[i + 1] - S[i]);
}

static inline double mask_val(const geom_t* g, int iy, int ix) {
  return g->mask ? (double)g->mask[(size_t)iy * g->XN + ix] : 1.0;
}

/* Per-ray constants of the forward kernel (MultiSlicesProjGPU.cu:120-158,
 * :176-181) for view angle th and channel u. */
typedef struct {
  int xmajor;          /* |cos| <= |sin|: integrate over x columns */
  double fL, fR;       /* boundary line slopes */
  double Lx, Ly, Rx, Ry;
  double cv;           /* dx / |dir component| */
} ray_t;

static inline void ray_setup(const geom_t* g, double cs, double sn, int u, ray_t* r) {
  const double sx = g->x0 * cs - g->y0 * sn, sy = g->x0 * sn + g->y0 * cs;
  const double xd = g->xds[u], yd = g->yds[u];
  const double Dx = xd * cs - yd * sn, Dy = xd * sn + yd * cs;
  r->Lx = g->bx[u] * cs - g->by[u] * sn;
  r->Ly = g->bx[u] * sn + g->by[u] * cs;
  r->Rx = g->bx[u + 1] * cs - g->by[u + 1] * sn;
  r->Ry = g->bx[u + 1] * sn + g->by[u + 1] * cs;
  double ddx = Dx - sx, ddy = Dy - sy;
  const double nrm = sqrt(ddx * ddx + ddy * ddy);
  ddx /= nrm; ddy /= nrm;
  r->xmajor = fabs(cs) <= fabs(sn);
  if (r->xmajor) {
    r->fL = (r->Ly - sy) / (r->Lx - sx);
    r->fR = (r->Ry - sy) / (r->Rx - sx);
    r->cv = g->dx / fabs(ddx);
  } else {
    r->fL = (r->Lx - sx) / (r->Ly - sy);
    r->fR = (r->Rx - sx) / (r->Ry - sy);
    r->cv = g->dx / fabs(ddy);
  }
}

/* Footprint of ray r on line ii: texel coordinates tL, tR of the two
 * boundary rays (MultiSlicesProjGPU.cu:161-168 / :184-191) and the
 * intersection length in mm. */
static inline void ray_line(const geom_t* g, const ray_t* r, int ii, double* tL, double* tR,
                            double* len) {
  if (r->xmajor) {
    const double obj = (ii - g->ocx) * g->dx;
    const double rL = (obj - r->Lx) * r->fL + r->Ly;
    const double rR = (obj - r->Rx) * r->fR + r->Ry;
    *len = rR - rL;
    *tL = rL / g->dx + g->ocy + 1.0;
    *tR = rR / g->dx + g->ocy + 1.0;
  } else {
    const double obj = (ii - g->ocy) * g->dx;
    const double rL = (obj - r->Ly) * r->fL + r->Lx;
    const double rR = (obj - r->Ry) * r->fR + r->Rx;
    *len = rR - rL;
    *tL = rL / g->dx + g->ocx + 1.0;
    *tR = rR / g->dx + g->ocx + 1.0;
  }
}

/* ---------------------------------------------------------------- forward */

/* Forward projection, double in / double out.
 * vol [YN][XN][SLN], angs [PN][SLN], prj [PN][DNU][SLN]. */
static int proj_d(const geom_t* g, const double* angs, int PN, int SLN, const double* vol,
                  double* prj, int nthreads) {
  const int XN = g->XN, YN = g->YN, DNU = g->DNU;
  const size_t wx = (size_t)(XN + 1), wy = (size_t)(YN + 1);
  /* SATx[z][y][x'] (x' = 0..XN), SATy[z][x][y'] (y' = 0..YN):
   * MultiSlicesProjGPU.cu:25-51 (ZXY / ZYX padded copies, prefix along x / y). */
  double* satx = (double*)malloc(sizeof(double) * SLN * YN * wx);
  double* saty = (double*)malloc(sizeof(double) * SLN * XN * wy);
  if (!satx || !saty) { free(satx); free(saty); return -1; }
  #pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int z = 0; z < SLN; ++z) {
    for (int y = 0; y < YN; ++y) {
      double* S = satx + ((size_t)z * YN + y) * wx;
      S[0] = 0.0;
      for (int x = 0; x < XN; ++x)
        S[x + 1] = S[x] + vol[((size_t)y * XN + x) * SLN + z] * mask_val(g, y, x);
    }
    for (int x = 0; x < XN; ++x) {
      double* S = saty + ((size_t)z * XN + x) * wy;
      S[0] = 0.0;
      for (int y = 0; y < YN; ++y)
        S[y + 1] = S[y] + vol[((size_t)y * XN + x) * SLN + z] * mask_val(g, y, x);
    }
  }
  #pragma omp parallel for collapse(2) num_threads(nthreads) schedule(dynamic)
  for (int p = 0; p < PN; ++p) {
    for (int z = 0; z < SLN; ++z) {
      const double th = wrap_angle(angs[(size_t)p * SLN + z]);
      const double cs = cos(th), sn = sin(th);
      for (int u = 0; u < DNU; ++u) {
        ray_t r;
        ray_setup(g, cs, sn, u, &r);
        double summ = 0.0;
        const int nl = r.xmajor ? XN : YN;
        for (int ii = 0; ii < nl; ++ii) {
          double tL, tR, len;
          ray_line(g, &r, ii, &tL, &tR, &len);
          const double* S;
          int W;
          if (r.xmajor) { S = saty + ((size_t)z * XN + ii) * wy; W = YN + 1; }
          else { S = satx + ((size_t)z * YN + ii) * wx; W = XN + 1; }
          summ += (sat_fetch(S, W, tR) - sat_fetch(S, W, tL)) / len;
        }
        prj[((size_t)p * DNU + u) * SLN + z] = summ * r.cv;
      }
    }
  }
  free(satx);
  free(saty);
  return 0;
}

/* ---------------------------------------------------------- REF back */

static double ref_dbeta(const geom_t* g) {
  /* MultiSlicesBackGPU.cu:211, :226-227 */
  const double S2D = hypot((double)g->xds[0] - g->x0, (double)g->yds[0] - g->y0);
  const double ex = (double)g->xds[1] - g->xds[0], ey = (double)g->yds[1] - g->yds[0];
  const double dts = sqrt(ex * ex + ey * ey);
  return atan(dts / S2D * 0.5) * 2.0;
}

/* Reference backprojector (MultiSlicesBackGPU.cu:115-184), double in/out.
 * prj [PN][DNU][SLN] -> vol [YN][XN][SLN]; masked voxels are 0. */
static int back_ref_d(const geom_t* g, double detCntIdx, const double* angs, int PN, int SLN,
                      const double* prj, double* vol, int nthreads) {
  const int XN = g->XN, YN = g->YN, DNU = g->DNU;
  const size_t W = (size_t)DNU + 1;
  double* sat = (double*)malloc(sizeof(double) * PN * SLN * W); /* [p][z][u'] */
  if (!sat) return -1;
  #pragma omp parallel for collapse(2) num_threads(nthreads) schedule(static)
  for (int p = 0; p < PN; ++p)
    for (int z = 0; z < SLN; ++z) {
      double* S = sat + ((size_t)p * SLN + z) * W;
      S[0] = 0.0;
      for (int u = 0; u < DNU; ++u) S[u + 1] = S[u] + prj[((size_t)p * DNU + u) * SLN + z];
    }
  const double dbeta = ref_dbeta(g);
  const double inv_sid = 1.0 / sqrt(g->x0 * g->x0 + g->y0 * g->y0);
  double* cs = (double*)malloc(sizeof(double) * PN * SLN * 2);
  if (!cs) { free(sat); return -1; }
  for (size_t i = 0; i < (size_t)PN * SLN; ++i) {
    const double th = wrap_angle(angs[i]);
    cs[2 * i] = cos(th);
    cs[2 * i + 1] = sin(th);
  }
  #pragma omp parallel for collapse(2) num_threads(nthreads) schedule(dynamic)
  for (int iy = 0; iy < YN; ++iy)
    for (int ix = 0; ix < XN; ++ix) {
      const int on = g->mask ? g->mask[(size_t)iy * XN + ix] != 0 : 1;
      for (int z = 0; z < SLN; ++z) {
        if (!on) { vol[((size_t)iy * XN + ix) * SLN + z] = 0.0; continue; }
        const double vx = (ix - g->ocx) * g->dx, vy = (iy - g->ocy) * g->dx;
        double summ = 0.0;
        for (int p = 0; p < PN; ++p) {
          const double c = cs[2 * ((size_t)p * SLN + z)], s = cs[2 * ((size_t)p * SLN + z) + 1];
          const double sx = g->x0 * c - g->y0 * s, sy = g->x0 * s + g->y0 * c;
          const double dx_ = vx - sx, dy_ = vy - sy;
          const double l2 = dx_ * dx_ + dy_ * dy_;
          const double linv = 1.0 / sqrt(l2);
          const double alpha = asin((sy * dx_ - sx * dy_) * inv_sid * linv);
          const double ddv = fabs(sx) > fabs(sy) ? dx_ : dy_;
          const double da = ddv / l2 * g->dx * 0.5;
          const double cosv = g->dx / ddv * sqrt(l2);
          const double iL = (alpha - da) / dbeta + detCntIdx + 1.0;
          const double iR = (alpha + da) / dbeta + detCntIdx + 1.0;
          const double* S = sat + ((size_t)p * SLN + z) * W;
          summ += (sat_fetch(S, (int)W, iR) - sat_fetch(S, (int)W, iL)) * cosv;
        }
        vol[((size_t)iy * XN + ix) * SLN + z] = summ;
      }
    }
  free(cs);
  free(sat);
  return 0;
}

/* ---------------------------------------------------------- ADJ back */

/* Weight of pixel k in the interpolated prefix sum at sample position c
 * (already clamped to [0, N]): clamp(c - k, 0, 1). */
static inline double ramp(double c, int k) {
  double v = c - (double)k;
  return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

static inline double clampc(double t, int N) {
  double c = t - 0.5;
  if (!(c > 0.0)) c = 0.0;
  if (c > (double)N) c = (double)N;
  return c;
}

/* Exact transpose of proj_d: prj [PN][DNU][SLN] -> vol [YN][XN][SLN]. */
static int back_adj_d(const geom_t* g, const double* angs, int PN, int SLN, const double* prj,
                      double* vol, int nthreads) {
  const int XN = g->XN, YN = g->YN, DNU = g->DNU;
  const size_t V = (size_t)XN * YN * SLN;
  int nt = nthreads > 0 ? nthreads : 1;
  double* acc = (double*)calloc((size_t)nt * V, sizeof(double));
  if (!acc) return -1;
  #pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* my = acc + (size_t)tid * V;
    #pragma omp for collapse(2) schedule(dynamic)
    for (int p = 0; p < PN; ++p)
      for (int z = 0; z < SLN; ++z) {
        const double th = wrap_angle(angs[(size_t)p * SLN + z]);
        const double cs = cos(th), sn = sin(th);
        for (int u = 0; u < DNU; ++u) {
          const double val = prj[((size_t)p * DNU + u) * SLN + z];
          if (val == 0.0) continue;
          ray_t r;
          ray_setup(g, cs, sn, u, &r);
          const int nl = r.xmajor ? XN : YN;
          const int N = r.xmajor ? YN : XN;
          for (int ii = 0; ii < nl; ++ii) {
            double tL, tR, len;
            ray_line(g, &r, ii, &tL, &tR, &len);
            const double cL = clampc(tL, N), cR = clampc(tR, N);
            const double lo = cL < cR ? cL : cR, hi = cL < cR ? cR : cL;
            int k0 = (int)floor(lo), k1 = (int)ceil(hi);
            if (k0 < 0) k0 = 0;
            if (k1 > N) k1 = N;
            const double wgt = val * r.cv / len;
            for (int k = k0; k < k1; ++k) {
              const double w = (ramp(cR, k) - ramp(cL, k)) * wgt;
              const size_t idx = r.xmajor ? ((size_t)k * XN + ii) : ((size_t)ii * XN + k);
              my[idx * SLN + z] += w;
            }
          }
        }
      }
  }
  #pragma omp parallel for num_threads(nt) schedule(static)
  for (size_t i = 0; i < (size_t)XN * YN; ++i) {
    const double m = g->mask ? (double)g->mask[i] : 1.0;
    for (int z = 0; z < SLN; ++z) {
      double s = 0.0;
      for (int t = 0; t < nt; ++t) s += acc[(size_t)t * V + i * SLN + z];
      vol[i * SLN + z] = s * m;
    }
  }
  free(acc);
  return 0;
}

/* ------------------------------------------------------------- public API */

static double* to_double(const float* a, size_t n) {
  double* d = (double*)malloc(sizeof(double) * (n ? n : 1));
  if (d)
    for (size_t i = 0; i < n; ++i) d[i] = a[i];
  return d;
}

/* Argument order of MultiSlicesProjGPU (MultiSlicesProjGPU.cu:552-567). */
int orc_proj(float x0, float y0, int DNU, const float* xds, const float* yds, float imgXCenter,
             float imgYCenter, const float* hangs, int PN, int XN, int YN, int SLN,
             const float* vol, float dx, const uint8_t* mask, double* prj, int nthreads) {
  geom_t g;
  if (geom_init(&g, x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, XN, YN, dx, mask)) return -1;
  double* a = to_double(hangs, (size_t)PN * SLN);
  double* v = to_double(vol, (size_t)XN * YN * SLN);
  int rc = (a && v) ? proj_d(&g, a, PN, SLN, v, prj, nthreads) : -1;
  free(a); free(v); geom_free(&g);
  return rc;
}

/* Argument order of MultiSlicesBackGPU (MultiSlicesBackGPU.cu:411-427);
 * mode 0 = REF (reference backprojector), 1 = ADJ (exact transpose). */
int orc_back(float x0, float y0, int DNU, const float* xds, const float* yds, float detCntIdx,
             float imgXCenter, float imgYCenter, const float* hangs, int PN, int XN, int YN,
             int SLN, const float* prj, float dx, const uint8_t* mask, int mode, double* vol,
             int nthreads) {
  geom_t g;
  if (geom_init(&g, x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, XN, YN, dx, mask)) return -1;
  double* a = to_double(hangs, (size_t)PN * SLN);
  double* q = to_double(prj, (size_t)PN * DNU * SLN);
  int rc = -1;
  if (a && q)
    rc = mode == 0 ? back_ref_d(&g, detCntIdx, a, PN, SLN, q, vol, nthreads)
                   : back_adj_d(&g, a, PN, SLN, q, vol, nthreads);
  free(a); free(q); geom_free(&g);
  return rc;
}

/* Double-precision entry points on already-double data (for OS-SART-style
 * callers that keep FP64 state). */
int orc_proj_d(float x0, float y0, int DNU, const float* xds, const float* yds, float imgXCenter,
               float imgYCenter, const double* angs, int PN, int XN, int YN, int SLN,
               const double* vol, float dx, const uint8_t* mask, double* prj, int nthreads) {
  geom_t g;
  if (geom_init(&g, x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, XN, YN, dx, mask)) return -1;
  int rc = proj_d(&g, angs, PN, SLN, vol, prj, nthreads);
  geom_free(&g);
  return rc;
}

int orc_back_d(float x0, float y0, int DNU, const float* xds, const float* yds, float detCntIdx,
               float imgXCenter, float imgYCenter, const double* angs, int PN, int XN, int YN,
               int SLN, const double* prj, float dx, const uint8_t* mask, int mode, double* vol,
               int nthreads) {
  geom_t g;
  if (geom_init(&g, x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, XN, YN, dx, mask)) return -1;
  int rc = mode == 0 ? back_ref_d(&g, detCntIdx, angs, PN, SLN, prj, vol, nthreads)
                     : back_adj_d(&g, angs, PN, SLN, prj, vol, nthreads);
  geom_free(&g);
  return rc;
}

/* OS-SART with optional FISTA momentum and non-negativity
 * (OSSART_AAPM.m:49-118), all state in double.
 *   hangs  [PNall][SLN] view angles, proj [PNall][DNU][SLN] measured sinogram,
 *   init   [YN][XN][SLN] initial image, out [YN][XN][SLN] result.
 * Subset k (0-based) holds views k, k + numOfOS, k + 2 numOfOS, ... (:60).
 * Row/column sums come from slice 0 and are reused for every slice (:61-64).
 * Where a row/column sum is 0 the value is left un-normalised (:88, :94).
 * nonneg != 0 clamps the image at 0 after every subset update (not in the
 * reference).  back_mode: 0 REF, 1 ADJ.  *iter_seconds (may be NULL) gets the
 * wall time of the iterations alone (weights excluded). */
int orc_ossart(float x0, float y0, int DNU, const float* xds, const float* yds, float detCntIdx,
               float imgXCenter, float imgYCenter, const float* hangs, int PNall, int XN, int YN,
               int SLN, const float* proj, const float* init, float dx, const uint8_t* mask,
               int numOfIter, int numOfOS, int useFISTA, int nonneg, int back_mode, double* out,
               int nthreads, double* iter_seconds) {
  geom_t g;
  if (numOfOS < 1 || numOfOS > PNall) return -2;
  if (geom_init(&g, x0, y0, DNU, xds, yds, imgXCenter, imgYCenter, XN, YN, dx, mask)) return -1;
  const size_t V = (size_t)XN * YN * SLN, NXY = (size_t)XN * YN;
  const int PNs_max = (PNall + numOfOS - 1) / numOfOS;
  double* x = out;
  double* last = (double*)malloc(sizeof(double) * V);
  double* angs = (double*)malloc(sizeof(double) * PNs_max * SLN);
  double* angs1 = (double*)malloc(sizeof(double) * PNs_max);
  double* ysub = (double*)malloc(sizeof(double) * (size_t)PNs_max * DNU * SLN);
  double* prj = (double*)malloc(sizeof(double) * (size_t)PNs_max * DNU * SLN);
  double* tp = (double*)malloc(sizeof(double) * V);
  double* rows = (double*)malloc(sizeof(double) * (size_t)numOfOS * PNs_max * DNU);
  double* cols = (double*)malloc(sizeof(double) * (size_t)numOfOS * NXY);
  double* ones = (double*)malloc(sizeof(double) * (NXY > (size_t)PNs_max * DNU ? NXY : (size_t)PNs_max * DNU));
  int rc = 0;
  if (!last || !angs || !angs1 || !ysub || !prj || !tp || !rows || !cols || !ones) { rc = -1; goto done; }
  for (size_t i = 0; i < V; ++i) x[i] = init[i];
  /* weights from slice 0 (OSSART_AAPM.m:59-66) */
  for (int k = 0; k < numOfOS; ++k) {
    int PNs = 0;
    for (int v = k; v < PNall; v += numOfOS) angs1[PNs++] = hangs[(size_t)v * SLN + 0];
    for (size_t i = 0; i < NXY; ++i) ones[i] = 1.0;
    if ((rc = proj_d(&g, angs1, PNs, 1, ones, rows + (size_t)k * PNs_max * DNU, nthreads))) goto done;
    for (size_t i = 0; i < (size_t)PNs * DNU; ++i) ones[i] = 1.0;
    if (back_mode == 0) rc = back_ref_d(&g, detCntIdx, angs1, PNs, 1, ones, cols + (size_t)k * NXY, nthreads);
    else rc = back_adj_d(&g, angs1, PNs, 1, ones, cols + (size_t)k * NXY, nthreads);
    if (rc) goto done;
  }
  double t0 = 1.0;
  double wall0 = 0.0;
#ifdef _OPENMP
  wall0 = omp_get_wtime();
#endif
  for (int it = 0; it < numOfIter; ++it) {
    if (useFISTA) memcpy(last, x, sizeof(double) * V);
    for (int k = 0; k < numOfOS; ++k) {
      int PNs = 0;
      for (int v = k; v < PNall; v += numOfOS, ++PNs) {
        for (int z = 0; z < SLN; ++z) angs[(size_t)PNs * SLN + z] = hangs[(size_t)v * SLN + z];
        for (size_t e = 0; e < (size_t)DNU * SLN; ++e)
          ysub[(size_t)PNs * DNU * SLN + e] = proj[(size_t)v * DNU * SLN + e];
      }
      if ((rc = proj_d(&g, angs, PNs, SLN, x, prj, nthreads))) goto done;
      const double* rs = rows + (size_t)k * PNs_max * DNU;
      for (size_t pu = 0; pu < (size_t)PNs * DNU; ++pu)
        if (rs[pu] != 0.0)
          for (int z = 0; z < SLN; ++z) {
            const size_t e = pu * SLN + z;
            prj[e] = (ysub[e] - prj[e]) / rs[pu];
          }
      if (back_mode == 0) rc = back_ref_d(&g, detCntIdx, angs, PNs, SLN, prj, tp, nthreads);
      else rc = back_adj_d(&g, angs, PNs, SLN, prj, tp, nthreads);
      if (rc) goto done;
      const double* cl = cols + (size_t)k * NXY;
      for (size_t i = 0; i < NXY; ++i)
        for (int z = 0; z < SLN; ++z) {
          const size_t e = i * SLN + z;
          double t = tp[e];
          if (cl[i] != 0.0) t /= cl[i];
          double v = x[e] + t;
          if (nonneg && v < 0.0) v = 0.0;
          x[e] = v;
        }
    }
    if (useFISTA) {
      const double t1 = (1.0 + sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;
      const double m = (t0 - 1.0) / t1;
      for (size_t e = 0; e < V; ++e) x[e] = x[e] + m * (x[e] - last[e]);
      t0 = t1;
    }
  }
  if (iter_seconds) {
#ifdef _OPENMP
    *iter_seconds = omp_get_wtime() - wall0;
#else
    *iter_seconds = 0.0;
#endif
  }
done:
  free(last); free(angs); free(angs1); free(ysub); free(prj); free(tp); free(rows); free(cols);
  free(ones);
  geom_free(&g);
  return rc;
}
