/*
 * xt_oracle.c -- CPU restatement of the reference TIMBIR engine's hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see xt_oracle.h).  Every routine names the
 * reference routine of gromitsun/timbir-python Source_Code_4D_Fast it
 * restates.  Arithmetic keeps the reference's C promotion order: where the
 * reference mixes a float (Real_t) with a double literal or a libm call, the
 * expression is evaluated in double and rounded once on assignment, exactly as
 * gcc does on x86-64 (SSE, no FMA contraction).  With that, the float build of
 * this file and the float build of the reference agree bit for bit, which the
 * tests check against oracle/_ref and tests/golden.
 */
#include "xt_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define XO_PROFILE_RES 1536   /* PROFILE_RESOLUTION, XT_Constants.h:123 */
#define XO_BEAM_RES 512       /* BEAM_RESOLUTION, XT_Constants.h:124 */
#define XO_HR_BINS 64         /* DETECTOR_RESPONSE_BINS, XT_Constants.h:125 */
#define XO_MRF_Q 2.0          /* MRF_Q, XT_Constants.h:109 */
#define XO_NHICD_ITERS 10     /* XT_Init.c:438 */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define XO_PI_2 1.57079632679489661923132169163975144
#define XO_PI_4 0.785398163397448309615660845819875721

struct xo_ctx {
  xo_params prm;
  int32_t N_r, N_t, N_p, N_x, N_y, N_z, N_time, nzb, zovl, amax;
  xo_real delta_r, delta_t, R0, RMax, T0, x0, y0, delta_xy, delta_z, mult_xy;
  xo_real OffsetR, MRF_P, C_S, C_T, alpha, Sigma_S_Q, Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P;
  xo_real SF[3][3][3], TF, T, delta, var_est, StopThreshold, radius_obj;
  xo_real *view, *time, *cosv, *sinv, *hr;
  int32_t *proj_num, *proj_start, *proj_idx;
  xo_real *y, *w, *d, *e;
  uint8_t *sel;
  xo_real *obj;      /* [N_time][N_z+2][N_y][N_x], slice 0 and N_z+1 are the unused halo */
  uint8_t *mask;     /* [N_time][N_y][N_x][N_z] */
  xo_real *magmap;   /* [N_time][nzb][N_y][N_x] */
  int32_t *xr, *yr, *xn, *yn, *usn, *nsn;
  /* z slab of a volume split over ranks: a neighbour below / above, whose
   * adjacent slice sits in halo slice 0 / N_z + 1 (XT_Init.c:290-294) */
  int32_t slab_lo, slab_hi;
};

#define OBJ(c, i, z, j, k) ((c)->obj[((((size_t)(i) * ((c)->N_z + 2) + (z)) * (c)->N_y + (j)) * (c)->N_x + (k))])
#define SIDX(c, p, r, t) ((((size_t)(p) * (c)->N_r + (r)) * (c)->N_t) + (t))

/* ---------------------------------------------------------------- RNG ----
 * Park-Miller LCG, randlib.c:119-141 (random2) and :168 (srandom2). */
static uint32_t xo_sd[2];
static long xo_tmp;

void xo_srandom2(uint32_t num) {
  xo_tmp = num;
  xo_sd[0] = (uint32_t)(xo_tmp >> 16);
  xo_sd[1] = (uint32_t)(xo_tmp & 0xffff);
}

double xo_random2(void) {
  xo_sd[1] *= 16807u;
  xo_sd[0] *= 16807u;
  xo_tmp = (long)((xo_sd[0] >> 15) + ((xo_sd[0] & 0x7fff) << 16));
  xo_tmp += (long)xo_sd[1];
  if (xo_tmp & 0x80000000L) {
    xo_tmp++;
    xo_tmp &= 0x7fffffffL;
  }
  xo_sd[0] = (uint32_t)(xo_tmp >> 16);
  xo_sd[1] = (uint32_t)(xo_tmp & 0xffff);
  return ((double)xo_tmp) / 2147483647.0;
}

/* ------------------------------------------------------------ geometry ---- */

/* distance2node, XT_Init.c:204-207 */
static xo_real xo_dist(int i, int j, int k, int l) {
  return (xo_real)sqrt(pow((xo_real)i - 1.0, 2.0) + pow((xo_real)j - 1.0, 2.0) +
                       pow((xo_real)k - 1.0, 2.0) + pow((xo_real)l - 1.0, 2.0));
}

/* initFilter, XT_Init.c:210-256 */
static void xo_init_filter(xo_ctx *c, xo_real delta_Rtime) {
  xo_real sum = 0, temp1, prior_const;
  prior_const = c->mult_xy * c->mult_xy * c->mult_xy * delta_Rtime;
  c->TF = (xo_real)(1.0 / xo_dist(0, 1, 1, 1));
  sum = (xo_real)(sum + 2.0 * c->TF);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        if (i != 1 || j != 1 || k != 1) {
          temp1 = (xo_real)(1.0 / xo_dist(1, i, j, k));
          c->SF[i][j][k] = temp1;
          sum = sum + temp1;
        } else {
          c->SF[i][j][k] = 0;
        }
      }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) c->SF[i][j][k] = prior_const * c->SF[i][j][k] / sum;
  c->TF = prior_const * c->TF / sum;
}

/* calculateVoxelProfile + initializeBeamProfile + DetectorResponseProfile,
 * XT_Profile.c:46-103, :107-123, :128-171 (H_r part only). */
static void xo_detector_response(xo_ctx *c) {
  xo_real *vp = (xo_real *)malloc(sizeof(xo_real) * (size_t)c->N_p * XO_PROFILE_RES);
  xo_real beam[XO_BEAM_RES];
  for (int i = 0; i < c->N_p; i++) {
    xo_real angle = c->view[i], maxv, temp, dist1, dist2, LC, LN, RN, RC, t;
    while (angle > XO_PI_2) angle = (xo_real)(angle - XO_PI_2);
    while (angle < 0) angle = (xo_real)(angle + XO_PI_2);
    if (angle <= XO_PI_4)
      maxv = (xo_real)(c->delta_xy / cos(angle));
    else
      maxv = (xo_real)(c->delta_xy / cos(XO_PI_2 - angle));
    temp = (xo_real)cos(XO_PI_4);
    dist1 = (xo_real)(temp * cos((XO_PI_4 - angle)));
    dist2 = (xo_real)(temp * fabs((cos((XO_PI_4 + angle)))));
    LC = 1 - dist1;
    LN = 1 - dist2;
    RN = 1 + dist2;
    RC = 1 + dist1;
    for (int j = 0; j < XO_PROFILE_RES; j++) {
      xo_real *o = &vp[(size_t)i * XO_PROFILE_RES + j];
      t = (xo_real)(2.0 * j / XO_PROFILE_RES);
      if (t <= LC || t >= RC)
        *o = 0;
      else if (t > RN)
        *o = maxv * (RC - t) / (RC - RN);
      else if (t >= LN)
        *o = maxv;
      else
        *o = maxv * (t - LC) / (LN - LC);
    }
  }
  xo_real bsum = 0;
  for (int i = 0; i < XO_BEAM_RES; i++) {
    beam[i] = (xo_real)(0.54 - 0.46 * cos((2 * M_PI / XO_BEAM_RES) * i));
    bsum = bsum + beam[i];
  }
  for (int i = 0; i < XO_BEAM_RES; i++) beam[i] /= bsum;

  xo_real r0 = -(c->delta_r) / 2;       /* BeamWidth = delta_r, XT_Init.c:378 */
  xo_real step = (c->delta_r) / XO_BEAM_RES;
  xo_real tconst = (XO_PROFILE_RES) / (2 * c->delta_xy);
  for (int k = 0; k < c->N_p; k++) {
    int i;
    for (i = 0; i < XO_HR_BINS; i++) {
      xo_real center = i * c->OffsetR;
      xo_real rmin = center - c->delta_xy;
      xo_real sum = 0;
      for (int p = 0; p < XO_BEAM_RES; p++) {
        xo_real r = r0 + p * step;
        int32_t pi = (int32_t)floor((r - rmin) * tconst);
        if (pi >= 0 && pi <= XO_PROFILE_RES - 1) sum += (vp[(size_t)k * XO_PROFILE_RES + pi] * beam[p]);
      }
      c->hr[(size_t)k * (XO_HR_BINS + 1) + i] = sum;
    }
    c->hr[(size_t)k * (XO_HR_BINS + 1) + i] = 0.0;
  }
  free(vp);
}

xo_ctx *xo_create(const xo_params *prm, const double *view_times, const double *view_angles_deg) {
  xo_ctx *c = (xo_ctx *)calloc(1, sizeof(xo_ctx));
  c->prm = *prm;
  /* argsParser, XT_Init.c:510-511, 542-589 */
  xo_real slope_HU = (xo_real)((1000 - 0) / (0.521225397034623 * 1.0 - 0.496372335005353 * 0.001205) / 0.0001);
  xo_real c_HU = (xo_real)(-slope_HU * (0.496372335005353 * 0.001205 * 0.0001));
  c->MRF_P = (xo_real)prm->p;
  xo_real Sigma_S = (xo_real)(prm->sigma_s - c_HU) / slope_HU;
  xo_real Sigma_T = (xo_real)(prm->sigma_t - c_HU) / slope_HU;
  c->C_S = (xo_real)prm->c_s;
  c->C_T = (xo_real)prm->c_t;
  xo_real mult_xy = (xo_real)prm->mult_xy, mult_z = (xo_real)prm->mult_z;
  xo_real Length_R = (xo_real)prm->length_r, Length_T = (xo_real)prm->length_t;
  xo_real RotCenter = (xo_real)prm->rot_center;
  c->alpha = (xo_real)prm->alpha;
  xo_real Rtime0 = (xo_real)prm->Rtime0, delta_Rtime = (xo_real)prm->Rtime_delta;
  c->T = (xo_real)prm->zingerT;
  c->delta = (xo_real)prm->zingerDel;
  c->var_est = (xo_real)prm->var_est;
  c->StopThreshold = (xo_real)prm->voxel_thresh;
  c->radius_obj = (xo_real)prm->radius_obj;
  c->N_r = prm->N_r;
  c->N_p = prm->N_p;
  c->N_time = prm->N_time;
  c->mult_xy = mult_xy;
  xo_real delta_xy = mult_xy, delta_z = mult_z; /* sinobin 1, XT_Init.c:619-621 */
  c->zovl = (int32_t)mult_z;

  /* initStructures, XT_Init.c:293-400 (single rank) */
  Length_T = Length_T / 1;
  c->N_t = prm->N_t / 1;
  if (c->N_t % (int32_t)delta_z != 0 || c->N_r % (int32_t)delta_xy != 0) {
    free(c);
    return NULL;
  }
  c->delta_r = Length_R / (c->N_r);
  c->delta_t = Length_T / (c->N_t);
  c->R0 = -RotCenter * c->delta_r;
  c->RMax = (c->N_r - RotCenter) * c->delta_r;
  c->T0 = (xo_real)(-Length_T / 2.0);
  c->N_x = (int32_t)(c->N_r / delta_xy);
  c->N_y = (int32_t)(c->N_r / delta_xy);
  c->N_z = (int32_t)(c->N_t / delta_z);
  c->delta_xy = delta_xy * c->delta_r;
  c->delta_z = delta_z * c->delta_t;
  c->x0 = c->R0;
  c->y0 = (xo_real)(-Length_R / 2.0);
  c->OffsetR = (xo_real)((c->delta_xy / sqrt(2.0) + c->delta_r / 2.0) / XO_HR_BINS);
  c->Sigma_S_Q = (xo_real)pow((Sigma_S * mult_xy), XO_MRF_Q);
  c->Sigma_S_Q_P = (xo_real)pow(Sigma_S * mult_xy, XO_MRF_Q - c->MRF_P);
  c->Sigma_T_Q = (xo_real)pow((Sigma_T * delta_Rtime), XO_MRF_Q);
  c->Sigma_T_Q_P = (xo_real)pow(Sigma_T * delta_Rtime, XO_MRF_Q - c->MRF_P);
  c->nzb = (int32_t)(2 * floor(prm->num_threads / c->N_time));
  if (c->nzb < 2)
    c->nzb = 2;
  else if (c->nzb > c->N_z)
    c->nzb = c->N_z;
  c->amax = (int32_t)ceil(3 * c->delta_xy / c->delta_r); /* AvgNumXElements, XT_VoxUpdate.c:109 */
  xo_init_filter(c, delta_Rtime);

  /* initSparseAnglesfrmFile / initSparseAnglesOfObject / calculateSinCos,
   * XT_Init.c:98-125, 130-162, 259-272 */
  c->view = (xo_real *)calloc(c->N_p, sizeof(xo_real));
  c->time = (xo_real *)calloc(c->N_p, sizeof(xo_real));
  c->cosv = (xo_real *)calloc(c->N_p, sizeof(xo_real));
  c->sinv = (xo_real *)calloc(c->N_p, sizeof(xo_real));
  for (int i = 0; i < c->N_p; i++) {
    c->view[i] = (xo_real)((xo_real)view_angles_deg[i] * M_PI / 180.0);
    c->time[i] = (xo_real)view_times[i];
    c->cosv[i] = (xo_real)cos(c->view[i]);
    c->sinv[i] = (xo_real)sin(c->view[i]);
  }
  c->proj_num = (int32_t *)calloc(c->N_time, sizeof(int32_t));
  c->proj_start = (int32_t *)calloc(c->N_time, sizeof(int32_t));
  c->proj_idx = (int32_t *)calloc(c->N_p > 0 ? c->N_p : 1, sizeof(int32_t));
  {
    int32_t frame = 0, num = 0, start = 0;
    xo_real t2 = Rtime0 + delta_Rtime;
    for (int i = 0; i < c->N_p; i++) {
      while (c->time[i] >= t2 && frame + 1 < c->N_time) {
        c->proj_start[frame] = start;
        c->proj_num[frame] = num;
        start += num;
        t2 += delta_Rtime;
        frame++;
        num = 0;
      }
      c->proj_idx[start + num] = i;
      num++;
    }
    c->proj_start[frame] = start;
    c->proj_num[frame] = num;
  }

  size_t ns = (size_t)c->N_p * c->N_r * c->N_t, nxy = (size_t)c->N_x * c->N_y;
  c->hr = (xo_real *)calloc((size_t)c->N_p * (XO_HR_BINS + 1), sizeof(xo_real));
  xo_detector_response(c);
  c->y = (xo_real *)calloc(ns, sizeof(xo_real));
  c->w = (xo_real *)calloc(ns, sizeof(xo_real));
  c->e = (xo_real *)calloc(ns, sizeof(xo_real));
  c->sel = (uint8_t *)calloc(ns, 1);
  memset(c->sel, 1, ns);
  c->d = (xo_real *)calloc((size_t)c->N_r * c->N_t, sizeof(xo_real));
  c->obj = (xo_real *)calloc((size_t)c->N_time * (c->N_z + 2) * nxy, sizeof(xo_real));
  c->mask = (uint8_t *)calloc((size_t)c->N_time * nxy * c->N_z, 1);
  c->magmap = (xo_real *)calloc((size_t)c->N_time * c->nzb * nxy, sizeof(xo_real));
  size_t nl = (size_t)c->N_time * c->nzb * nxy;
  c->xr = (int32_t *)calloc(nl, 4);
  c->yr = (int32_t *)calloc(nl, 4);
  c->xn = (int32_t *)calloc(nl, 4);
  c->yn = (int32_t *)calloc(nl, 4);
  c->usn = (int32_t *)calloc((size_t)c->N_time * c->nzb, 4);
  c->nsn = (int32_t *)calloc((size_t)c->N_time * c->nzb, 4);

  /* object-support mask, XT_ICD_update.c:958-974 */
  for (int i = 0; i < c->N_time; i++)
    for (int j = 0; j < c->N_y; j++)
      for (int k = 0; k < c->N_x; k++) {
        xo_real x = (xo_real)(c->x0 + ((xo_real)k + 0.5) * c->delta_xy);
        xo_real y = (xo_real)(c->y0 + ((xo_real)j + 0.5) * c->delta_xy);
        uint8_t m = (x * x + y * y < c->radius_obj * c->radius_obj) ? 1 : 0;
        for (int l = 0; l < c->N_z; l++) c->mask[(((size_t)i * c->N_y + j) * c->N_x + k) * c->N_z + l] = m;
      }
  return c;
}

void xo_destroy(xo_ctx *c) {
  if (!c) return;
  free(c->view); free(c->time); free(c->cosv); free(c->sinv); free(c->hr);
  free(c->proj_num); free(c->proj_start); free(c->proj_idx);
  free(c->y); free(c->w); free(c->e); free(c->sel); free(c->d); free(c->obj);
  free(c->mask); free(c->magmap); free(c->xr); free(c->yr); free(c->xn); free(c->yn);
  free(c->usn); free(c->nsn);
  free(c);
}

void xo_dims(const xo_ctx *c, int32_t *d) {
  d[XO_NX] = c->N_x; d[XO_NY] = c->N_y; d[XO_NZ] = c->N_z; d[XO_NTIME] = c->N_time;
  d[XO_NR] = c->N_r; d[XO_NT] = c->N_t; d[XO_NP] = c->N_p; d[XO_NZB] = c->nzb; d[XO_ZOVL] = c->zovl;
}

void xo_derived(const xo_ctx *c, double *o) {
  o[0] = c->delta_r; o[1] = c->delta_t; o[2] = c->R0; o[3] = c->RMax; o[4] = c->x0; o[5] = c->y0;
  o[6] = c->delta_xy; o[7] = c->OffsetR; o[8] = c->Sigma_S_Q; o[9] = c->Sigma_S_Q_P;
  o[10] = c->Sigma_T_Q; o[11] = c->Sigma_T_Q_P; o[12] = c->TF;
  for (int i = 0; i < 27; i++) o[13 + i] = (&c->SF[0][0][0])[i];
}

void xo_views(const xo_ctx *c, xo_real *v, xo_real *cs, xo_real *sn, int32_t *pn, int32_t *pi) {
  for (int i = 0; i < c->N_p; i++) { v[i] = c->view[i]; cs[i] = c->cosv[i]; sn[i] = c->sinv[i]; pi[i] = c->proj_idx[i]; }
  for (int i = 0; i < c->N_time; i++) pn[i] = c->proj_num[i];
}

void xo_get_hr(const xo_ctx *c, xo_real *hr) { memcpy(hr, c->hr, sizeof(xo_real) * (size_t)c->N_p * (XO_HR_BINS + 1)); }

/* calcAMatrixColumnforAngle, XT_AMatrix.c:50-110 */
int32_t xo_amatrix(const xo_ctx *c, int32_t row, int32_t col, int32_t p, xo_real *vals, int32_t *idx) {
  xo_real x = (xo_real)(c->x0 + ((xo_real)col + 0.5) * c->delta_xy);
  xo_real y = (xo_real)(c->y0 + ((xo_real)row + 0.5) * c->delta_xy);
  xo_real r = x * c->cosv[p] - y * c->sinv[p];
  xo_real rmin = r - c->delta_xy, rmax = r + c->delta_xy;
  int32_t count = 0;
  if (rmax < c->R0 || rmin > c->RMax) return 0;
  int32_t imin = (int32_t)(floor(((rmin - c->R0) / c->delta_r)));
  int32_t imax = (int32_t)(floor((rmax - c->R0) / c->delta_r));
  if (imax >= c->N_r) imax = c->N_r - 1;
  if (imin < 0) imin = 0;
  const xo_real *H = &c->hr[(size_t)p * (XO_HR_BINS + 1)];
  for (int32_t j = imin; j <= imax; j++) {
    xo_real Rc = (xo_real)(c->R0 + (((xo_real)j) + 0.5) * (c->delta_r));
    xo_real dr = (xo_real)fabs(r - Rc);
    int32_t id = (int32_t)(floor((dr / c->OffsetR)));
    if (id >= 0 && id < XO_HR_BINS) {
      xo_real w1 = dr - id * c->OffsetR;
      xo_real w2 = c->OffsetR - w1;
      xo_real f1 = (w2 * H[id] + w1 * H[id + 1]) / c->OffsetR;
      if (f1 > 0) {
        vals[count] = f1;
        idx[count] = j;
        count++;
      }
    }
  }
  return count;
}

/* ---------------------------------------------------------- data access -- */
void xo_set_sino(xo_ctx *c, const xo_real *y, const xo_real *w, const xo_real *d) {
  size_t ns = (size_t)c->N_p * c->N_r * c->N_t;
  memcpy(c->y, y, ns * sizeof(xo_real));
  /* computeWriteSinogram, XT_Engine.c:115-118 */
  for (size_t i = 0; i < ns; i++) c->w[i] = w[i] / c->var_est;
  if (d)
    memcpy(c->d, d, (size_t)c->N_r * c->N_t * sizeof(xo_real));
  else
    memset(c->d, 0, (size_t)c->N_r * c->N_t * sizeof(xo_real));
}

void xo_set_object(xo_ctx *c, const xo_real *x) {
  size_t nxy = (size_t)c->N_x * c->N_y;
  for (int i = 0; i < c->N_time; i++)
    for (int z = 0; z < c->N_z; z++)
      memcpy(&OBJ(c, i, z + 1, 0, 0), &x[((size_t)i * c->N_z + z) * nxy], nxy * sizeof(xo_real));
}

void xo_get_object(const xo_ctx *c, xo_real *x) {
  size_t nxy = (size_t)c->N_x * c->N_y;
  for (int i = 0; i < c->N_time; i++)
    for (int z = 0; z < c->N_z; z++)
      memcpy(&x[((size_t)i * c->N_z + z) * nxy], &OBJ(c, i, z + 1, 0, 0), nxy * sizeof(xo_real));
}

void xo_get_error_sino(const xo_ctx *c, xo_real *e) { memcpy(e, c->e, sizeof(xo_real) * (size_t)c->N_p * c->N_r * c->N_t); }
void xo_get_weight(const xo_ctx *c, xo_real *w) { memcpy(w, c->w, sizeof(xo_real) * (size_t)c->N_p * c->N_r * c->N_t); }
void xo_get_offset(const xo_ctx *c, xo_real *d) { memcpy(d, c->d, sizeof(xo_real) * (size_t)c->N_r * c->N_t); }
xo_real xo_get_var(const xo_ctx *c) { return c->var_est; }
void xo_get_magmap(const xo_ctx *c, xo_real *m) {
  memcpy(m, c->magmap, sizeof(xo_real) * (size_t)c->N_time * c->nzb * c->N_x * c->N_y);
}
void xo_set_magmap(xo_ctx *c, const xo_real *m) {
  memcpy(c->magmap, m, sizeof(xo_real) * (size_t)c->N_time * c->nzb * c->N_x * c->N_y);
}

static inline uint8_t xo_select(const xo_ctx *c, xo_real e, xo_real w) {
  return (fabs(e * sqrt(w)) < c->T) ? 1 : 0;
}

void xo_set_error_sino(xo_ctx *c, const xo_real *e) {
  size_t ns = (size_t)c->N_p * c->N_r * c->N_t;
  memcpy(c->e, e, ns * sizeof(xo_real));
  for (size_t i = 0; i < ns; i++) c->sel[i] = xo_select(c, c->e[i], c->w[i]);
}

/* ------------------------------------------------- forward projection ---- */
/* initErrorSinogam first half + forward_project_voxel_AMat1D,
 * XT_ICD_update.c:551-569, XT_ForwardProject.c:8-25 */
/* Each view's sinogram entries receive their terms in the reference's
 * (row, column) order, so running the views on separate threads changes no
 * bit of the result. */
void xo_forward_project(const xo_ctx *c, xo_real *ax) {
  memset(ax, 0, sizeof(xo_real) * (size_t)c->N_p * c->N_r * c->N_t);
  for (int i = 0; i < c->N_time; i++) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int pp = 0; pp < c->proj_num[i]; pp++) {
      xo_real vals[16];
      int32_t idx[16];
      const int32_t p = c->proj_idx[c->proj_start[i] + pp];
      for (int j = 0; j < c->N_y; j++)
        for (int k = 0; k < c->N_x; k++) {
          int32_t cnt = xo_amatrix(c, j, k, p, vals, idx);
          for (int s = 0; s < c->N_z; s++) {
            xo_real pix = OBJ(c, i, s + 1, j, k);
            for (int m = 0; m < cnt; m++)
              for (int n = 0; n < c->zovl; n++) ax[SIDX(c, p, idx[m], s * c->zovl + n)] += pix * vals[m];
          }
        }
    }
  }
}

/* initErrorSinogam, XT_ICD_update.c:538-597 */
void xo_init_error_sino(xo_ctx *c) {
  size_t ns = (size_t)c->N_p * c->N_r * c->N_t;
  xo_forward_project(c, c->e);
  for (int p = 0; p < c->N_p; p++)
    for (int r = 0; r < c->N_r; r++)
      for (int t = 0; t < c->N_t; t++) {
        size_t q = SIDX(c, p, r, t);
        c->e[q] = c->y[q] - c->e[q] - c->d[(size_t)r * c->N_t + t];
        c->sel[q] = xo_select(c, c->e[q], c->w[q]);
      }
  (void)ns;
}

/* e = y - delta_t A x - d: the error sinogram of the matrix the voxel update
 * subtracts (A * delta_t, XT_VoxUpdate.c:27, 67), which the reference carries
 * from its zero start; initErrorSinogam's projector leaves delta_t out
 * (XT_ForwardProject.c:17).  Equal to xo_init_error_sino when delta_t = 1. */
void xo_init_error_sino_model(xo_ctx *c) {
  xo_forward_project(c, c->e);
  for (int p = 0; p < c->N_p; p++)
    for (int r = 0; r < c->N_r; r++)
      for (int t = 0; t < c->N_t; t++) {
        size_t q = SIDX(c, p, r, t);
        c->e[q] = c->y[q] - c->delta_t * c->e[q] - c->d[(size_t)r * c->N_t + t];
        c->sel[q] = xo_select(c, c->e[q], c->w[q]);
      }
}

/* ------------------------------------------------------------ prior ------ */
/* CE_QGGMRF_Spatial_Value / Temporal_Value, XT_ICD_update.c:79-87 */
static xo_real xo_qggmrf_value(const xo_ctx *c, xo_real delta, xo_real sq, xo_real sqp, xo_real cc) {
  return (xo_real)((pow(fabs(delta), XO_MRF_Q) / sq) / (cc + pow(fabs(delta), XO_MRF_Q - c->MRF_P) / sqp));
}

/* CE_QGGMRF_Spatial_Derivative / Temporal_Derivative, XT_ICD_update.c:89-115 */
static xo_real xo_qggmrf_deriv(const xo_ctx *c, xo_real delta, xo_real sq, xo_real sqp, xo_real cc) {
  xo_real temp1, temp2, temp3;
  temp1 = (xo_real)(pow(fabs(delta), XO_MRF_Q - c->MRF_P) / (sqp));
  temp2 = (xo_real)pow(fabs(delta), XO_MRF_Q - 1);
  temp3 = cc + temp1;
  if (delta < 0)
    return (xo_real)((-1 * temp2 / (temp3 * sq)) * (XO_MRF_Q - ((XO_MRF_Q - c->MRF_P) * temp1) / (temp3)));
  return (xo_real)((temp2 / (temp3 * sq)) * (XO_MRF_Q - ((XO_MRF_Q - c->MRF_P) * temp1) / (temp3)));
}

/* CE_FunctionalSubstitution, XT_ICD_update.c:130-179.  nhood/flags are in
 * [z][y][x] order of the 3x3x3 neighbourhood, tnhood = {t-1, t+1}. */
xo_real xo_functional_substitution(const xo_ctx *c, xo_real V, xo_real th1, xo_real th2,
                                   const xo_real *nh, const xo_real *tnh,
                                   const uint8_t *fl, const uint8_t *tfl) {
  xo_real u, temp1 = 0, temp2 = 0, temp_const, ref = V, d0, qp;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        int q = (i * 3 + j) * 3 + k;
        if (fl[q] && (i != 1 || j != 1 || k != 1)) {
          d0 = (ref - nh[q]);
          if (d0 != 0)
            qp = xo_qggmrf_deriv(c, d0, c->Sigma_S_Q, c->Sigma_S_Q_P, c->C_S) / (d0);
          else
            qp = (xo_real)(XO_MRF_Q / (c->Sigma_S_Q * c->C_S));
          temp_const = c->SF[i][j][k] * qp;
          temp1 += temp_const * nh[q];
          temp2 += temp_const;
        }
      }
  for (int i = 0; i < 2; i++) {
    if (tfl[i]) {
      d0 = (ref - tnh[i]);
      if (d0 != 0)
        qp = xo_qggmrf_deriv(c, d0, c->Sigma_T_Q, c->Sigma_T_Q_P, c->C_T) / (d0);
      else
        qp = (xo_real)(XO_MRF_Q / (c->Sigma_T_Q * c->C_T));
      temp_const = c->TF * qp;
      temp1 += temp_const * tnh[i];
      temp2 += temp_const;
    }
  }
  u = (temp1 + (th2 * V) - th1) / (temp2 + th2);
  ref = ref + c->alpha * (u - ref);
  if (c->prm.positivity && ref <= 0) ref = 0;
  return ref;
}

/* ------------------------------------------------------------- cost ------ */
/* computeCost, XT_ICD_update.c:181-314 (single rank, sequential order) */
xo_real xo_cost(xo_ctx *c, xo_real *fwd_out, xo_real *prior_out) {
  xo_real cost = 0, temp = 0, delta, forward, prior;
  for (int i = 0; i < c->N_p; i++)
    for (int j = 0; j < c->N_r; j++)
      for (int k = 0; k < c->N_t; k++) {
        size_t q = SIDX(c, i, j, k);
        temp = (xo_real)(c->e[q] * sqrt(c->w[q]));
        if (c->sel[q])
          temp = temp * temp;
        else
          temp = (xo_real)(2.0 * c->delta * c->T * fabs(temp) + c->T * c->T * (1.0 - 2.0 * c->delta));
        cost += temp;
      }
  cost /= 2.0;
  temp = 0;
  /* ranks other than the last include the pairs into the halo above, XT_ICD_update.c:203-205 */
  int Nz = c->slab_hi ? c->N_z + 2 : c->N_z + 1;
  const xo_real sq = c->Sigma_S_Q, sqp = c->Sigma_S_Q_P;
#define XO_SV(d) xo_qggmrf_value(c, (d), sq, sqp, c->C_S)
  for (int i = 0; i < c->N_time; i++)
    for (int p = 1; p < c->N_z + 1; p++)
      for (int j = 0; j < c->N_y; j++)
        for (int k = 0; k < c->N_x; k++) {
          int jm = j - 1 >= 0, km = k - 1 >= 0, pp = p + 1 < Nz, ip = i + 1 < c->N_time;
          int jp = j + 1 < c->N_y, kp = k + 1 < c->N_x;
          xo_real v = OBJ(c, i, p, j, k);
          if (kp) { delta = v - OBJ(c, i, p, j, k + 1); temp += c->SF[1][1][2] * XO_SV(delta); }
          if (jp) {
            if (km) { delta = v - OBJ(c, i, p, j + 1, k - 1); temp += c->SF[1][2][0] * XO_SV(delta); }
            delta = v - OBJ(c, i, p, j + 1, k); temp += c->SF[1][2][1] * XO_SV(delta);
            if (kp) { delta = v - OBJ(c, i, p, j + 1, k + 1); temp += c->SF[1][2][2] * XO_SV(delta); }
          }
          if (pp) {
            if (jm) { delta = v - OBJ(c, i, p + 1, j - 1, k); temp += c->SF[2][0][1] * XO_SV(delta); }
            delta = v - OBJ(c, i, p + 1, j, k); temp += c->SF[2][1][1] * XO_SV(delta);
            if (jp) { delta = v - OBJ(c, i, p + 1, j + 1, k); temp += c->SF[2][2][1] * XO_SV(delta); }
            if (jm) {
              if (km) { delta = v - OBJ(c, i, p + 1, j - 1, k - 1); temp += c->SF[2][0][0] * XO_SV(delta); }
              if (kp) { delta = v - OBJ(c, i, p + 1, j - 1, k + 1); temp += c->SF[2][0][2] * XO_SV(delta); }
            }
            if (km) { delta = v - OBJ(c, i, p + 1, j, k - 1); temp += c->SF[2][1][0] * XO_SV(delta); }
            if (jp) {
              if (km) { delta = v - OBJ(c, i, p + 1, j + 1, k - 1); temp += c->SF[2][2][0] * XO_SV(delta); }
              if (kp) { delta = v - OBJ(c, i, p + 1, j + 1, k + 1); temp += c->SF[2][2][2] * XO_SV(delta); }
            }
            if (kp) { delta = v - OBJ(c, i, p + 1, j, k + 1); temp += c->SF[2][1][2] * XO_SV(delta); }
          }
          if (ip) {
            delta = v - OBJ(c, i + 1, p, j, k);
            temp += c->TF * xo_qggmrf_value(c, delta, c->Sigma_T_Q, c->Sigma_T_Q_P, c->C_T);
          }
        }
#undef XO_SV
  forward = cost;
  prior = temp;
  forward = (xo_real)(forward + (xo_real)1 * (xo_real)c->N_p * (xo_real)c->N_r * (xo_real)c->N_t * log(c->var_est) / 2);
  if (fwd_out) *fwd_out = forward;
  if (prior_out) *prior_out = prior;
  return forward + prior;
}

/* The MAP cost of the current object with every sum in FP64: e64 =
 * y - delta_t A x - d from products of this build's A entries (FP32 in the
 * float build, as the reference's default build computes them), the data
 * term of computeCost (XT_ICD_update.c:181-200) on e64, and the prior over
 * the same forward neighbour pairs (XT_ICD_update.c:201-294) with this
 * build's constants promoted to FP64.  In the float build that is the
 * arithmetic of the GPU's FP64 MAP cost, term for term; the double build is
 * the reference's -DREAL_IS_DOUBLE evaluation (A itself in FP64). */
double xo_map_cost_fp64(const xo_ctx *c, double *fwd_out, double *prior_out) {
  const size_t ns = (size_t)c->N_p * c->N_r * c->N_t;
  double *ax = (double *)calloc(ns, sizeof(double));
  if (!ax) return NAN;
  for (int i = 0; i < c->N_time; i++) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int pp = 0; pp < c->proj_num[i]; pp++) {
      xo_real vals[16];
      int32_t idx[16];
      const int32_t p = c->proj_idx[c->proj_start[i] + pp];
      for (int j = 0; j < c->N_y; j++)
        for (int k = 0; k < c->N_x; k++) {
          int32_t cnt = xo_amatrix(c, j, k, p, vals, idx);
          for (int s = 0; s < c->N_z; s++) {
            const double pix = (double)OBJ(c, i, s + 1, j, k);
            for (int m = 0; m < cnt; m++)
              for (int n = 0; n < c->zovl; n++) ax[SIDX(c, p, idx[m], s * c->zovl + n)] += pix * (double)vals[m];
          }
        }
    }
  }
  const double T = (double)c->T, dl = (double)c->delta, dt = (double)c->delta_t;
  double data = 0;
#pragma omp parallel for reduction(+ : data)
  for (int p = 0; p < c->N_p; p++)
    for (int r = 0; r < c->N_r; r++)
      for (int t = 0; t < c->N_t; t++) {
        const size_t q = SIDX(c, p, r, t);
        const double e = (double)c->y[q] - dt * ax[q] - (double)c->d[(size_t)r * c->N_t + t];
        const double sw = e * sqrt((double)c->w[q]);
        data += fabs(sw) < T ? sw * sw : 2.0 * dl * T * fabs(sw) + T * T * (1.0 - 2.0 * dl);
      }
  free(ax);
  const double sq = (double)c->Sigma_S_Q, sqp = (double)c->Sigma_S_Q_P, cs = (double)c->C_S;
  const double tq = (double)c->Sigma_T_Q, tqp = (double)c->Sigma_T_Q_P, ct = (double)c->C_T, mp = (double)c->MRF_P;
  double prior = 0;
#pragma omp parallel for reduction(+ : prior)
  for (int p = 1; p < c->N_z + 1; p++)
    for (int i = 0; i < c->N_time; i++)
      for (int j = 0; j < c->N_y; j++)
        for (int k = 0; k < c->N_x; k++) {
          const double v = (double)OBJ(c, i, p, j, k);
          for (int dz = 0; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dx = -1; dx <= 1; dx++) {
                /* the 13 forward pairs: +x in the row, the next row, the next slice */
                if (dz == 0 && (dy < 0 || (dy == 0 && dx <= 0))) continue;
                const int jj = j + dy, kk = k + dx, zz = p + dz;
                if (jj < 0 || jj >= c->N_y || kk < 0 || kk >= c->N_x || zz > c->N_z + (c->slab_hi ? 1 : 0)) continue;
                const double a = fabs(v - (double)OBJ(c, i, zz, jj, kk));
                prior += (double)c->SF[1 + dz][1 + dy][1 + dx] * ((a * a / sq) / (cs + pow(a, 2.0 - mp) / sqp));
              }
          if (i + 1 < c->N_time) {
            const double a = fabs(v - (double)OBJ(c, i + 1, p, j, k));
            prior += (double)c->TF * ((a * a / tq) / (ct + pow(a, 2.0 - mp) / tqp));
          }
        }
  const double fwd = data / 2.0 + (double)c->N_p * c->N_r * c->N_t * log((double)c->var_est) / 2.0;
  if (fwd_out) *fwd_out = fwd;
  if (prior_out) *prior_out = prior;
  return fwd + prior;
}

/* ------------------------------------------------------------ slabs ----- */
void xo_set_slab(xo_ctx *c, int32_t below, int32_t above) {
  c->slab_lo = below;
  c->slab_hi = above;
}

/* this slab's boundary slices (1 and N_z of the haloed array), each
 * [N_time][N_y][N_x] -- what MPI_Send_Recv_Z_Slices sends, XT_MPI.c:47-81 */
void xo_get_boundary(const xo_ctx *c, xo_real *lo, xo_real *hi) {
  const size_t pl = (size_t)c->N_y * c->N_x;
  for (int i = 0; i < c->N_time; i++) {
    if (lo) memcpy(lo + i * pl, &OBJ(c, i, 1, 0, 0), pl * sizeof(xo_real));
    if (hi) memcpy(hi + i * pl, &OBJ(c, i, c->N_z, 0, 0), pl * sizeof(xo_real));
  }
}

/* the neighbours' slices into halo slices 0 and N_z + 1 (NULL: unchanged) */
void xo_set_halo(xo_ctx *c, const xo_real *lo, const xo_real *hi) {
  const size_t pl = (size_t)c->N_y * c->N_x;
  for (int i = 0; i < c->N_time; i++) {
    if (lo) memcpy(&OBJ(c, i, 0, 0, 0), lo + i * pl, pl * sizeof(xo_real));
    if (hi) memcpy(&OBJ(c, i, c->N_z + 1, 0, 0), hi + i * pl, pl * sizeof(xo_real));
  }
}

/* ------------------------------------------------------ voxel update ----- */
/* compute_voxel_update_Aditya, XT_VoxUpdate.c:11-83 */
static void xo_voxel_update(xo_ctx *c, const xo_real *av, const int32_t *ai, const int32_t *ac,
                            const xo_real *nh, const xo_real *tnh, const uint8_t *fl, const uint8_t *tfl,
                            int32_t i, int32_t slice, int32_t j, int32_t k) {
  xo_real V = OBJ(c, i, slice + 1, j, k), th1 = 0, th2 = 0, ts, pe;
  for (int pp = 0; pp < c->proj_num[i]; pp++) {
    int32_t p = c->proj_idx[c->proj_start[i] + pp];
    for (int q = 0; q < ac[pp]; q++) {
      int32_t ir = ai[pp * c->amax + q];
      pe = (av[pp * c->amax + q] * c->delta_t);
      for (int r = 0; r < c->zovl; r++) {
        size_t s = SIDX(c, p, ir, slice * c->zovl + r);
        if (c->sel[s]) {
          th2 += (pe * pe * c->w[s]);
          th1 += -(c->e[s] * pe * c->w[s]);
        } else {
          ts = (xo_real)(c->T * c->delta * sqrt(c->w[s]) / fabs(c->e[s]));
          th2 += (pe * pe * ts);
          th1 += -(c->e[s] * pe * ts);
        }
      }
    }
  }
  xo_real nv = xo_functional_substitution(c, V, th1, th2, nh, tnh, fl, tfl);
  OBJ(c, i, slice + 1, j, k) = nv;
  for (int pp = 0; pp < c->proj_num[i]; pp++) {
    int32_t p = c->proj_idx[c->proj_start[i] + pp];
    for (int q = 0; q < ac[pp]; q++) {
      int32_t ir = ai[pp * c->amax + q];
      pe = (av[pp * c->amax + q] * c->delta_t);
      for (int r = 0; r < c->zovl; r++) {
        size_t s = SIDX(c, p, ir, slice * c->zovl + r);
        c->e[s] -= (pe * (OBJ(c, i, slice + 1, j, k) - V));
        c->sel[s] = xo_select(c, c->e[s], c->w[s]);
      }
    }
  }
}

/* updateVoxels_Aditya, XT_VoxUpdate.c:85-254 (single rank: z_min=1, z_max=N_z) */
static xo_real xo_update_voxels(xo_ctx *c, int32_t i, int32_t zb, int32_t ze, int32_t xyb, int32_t xye,
                                const int32_t *xs, const int32_t *ys, int32_t iter, long *zero_count,
                                xo_real *mag) {
  xo_real total = 0, nh[27], tnh[2];
  uint8_t fl[27], tfl[2];
  int32_t maxv = 0;
  for (int t = 0; t < c->N_time; t++) maxv = c->proj_num[t] > maxv ? c->proj_num[t] : maxv;
  xo_real *av = (xo_real *)calloc((size_t)(maxv ? maxv : 1) * c->amax, sizeof(xo_real));
  int32_t *ai = (int32_t *)calloc((size_t)(maxv ? maxv : 1) * c->amax, 4);
  int32_t *ac = (int32_t *)calloc((size_t)(maxv ? maxv : 1), 4);
  /* a rank reads the halo slices of its neighbours, XT_VoxUpdate.c:94-99 */
  const int32_t zmin = c->slab_lo ? 0 : 1, zmax = c->slab_hi ? c->N_z + 1 : c->N_z;
  for (int32_t ix = xyb; ix <= xye; ix++) {
    int32_t k = xs[ix], j = ys[ix];
    mag[(size_t)j * c->N_x + k] = 0;
    for (int pp = 0; pp < c->proj_num[i]; pp++)
      ac[pp] = xo_amatrix(c, j, k, c->proj_idx[c->proj_start[i] + pp], &av[pp * c->amax], &ai[pp * c->amax]);
    for (int32_t s = zb; s <= ze; s++) {
      if (c->mask[(((size_t)i * c->N_y + j) * c->N_x + k) * c->N_z + s] != 1) continue;
      if (i - 1 >= 0) { tnh[0] = OBJ(c, i - 1, s + 1, j, k); tfl[0] = 1; } else { tnh[0] = 0; tfl[0] = 0; }
      if (i + 1 < c->N_time) { tnh[1] = OBJ(c, i + 1, s + 1, j, k); tfl[1] = 1; } else { tnh[1] = 0; tfl[1] = 0; }
      for (int p = 0; p < 3; p++) {
        int32_t ip = s + p;
        for (int q = 0; q < 3; q++) {
          int32_t iq = j + q - 1;
          for (int r = 0; r < 3; r++) {
            int32_t irr = k + r - 1, n = (p * 3 + q) * 3 + r;
            if (ip >= zmin && ip <= zmax && iq >= 0 && iq < c->N_y && irr >= 0 && irr < c->N_x) {
              nh[n] = OBJ(c, i, ip, iq, irr);
              fl[n] = 1;
            } else {
              nh[n] = 0;
              fl[n] = 0;
            }
          }
        }
      }
      nh[13] = 0.0;
      xo_real V = OBJ(c, i, s + 1, j, k);
      int zs = 0;
      if (V == 0.0 && iter > 1) { /* ZERO_SKIPPING, XT_VoxUpdate.c:208-232 */
        zs = 1;
        if (tnh[0] > 0.0 || tnh[1] > 0.0) zs = 0;
        for (int n = 0; n < 27; n++)
          if (nh[n] > 0.0) { zs = 0; break; }
      }
      if (!zs) {
        xo_voxel_update(c, av, ai, ac, nh, tnh, fl, tfl, i, s, j, k);
        mag[(size_t)j * c->N_x + k] = (xo_real)(mag[(size_t)j * c->N_x + k] + fabs(OBJ(c, i, s + 1, j, k) - V));
        total = (xo_real)(total + fabs(OBJ(c, i, s + 1, j, k)));
      } else {
        (*zero_count)++;
      }
    }
  }
  free(av); free(ai); free(ac);
  return total;
}

/* randomly_select_x_y, XT_ICD_update.c:599-631 */
void xo_random_lists(xo_ctx *c, int32_t *usn, int32_t *xsel, int32_t *ysel) {
  int32_t nxy = c->N_x * c->N_y;
  int32_t *counter = (int32_t *)malloc(sizeof(int32_t) * (size_t)nxy);
  for (int i = 0; i < c->N_time; i++)
    for (int b = 0; b < c->nzb; b++) {
      int32_t size = nxy, *u = &usn[i * c->nzb + b];
      int32_t *xl = &xsel[((size_t)i * c->nzb + b) * nxy], *yl = &ysel[((size_t)i * c->nzb + b) * nxy];
      for (int32_t q = 0; q < size; q++) counter[q] = q;
      *u = 0;
      for (int32_t jj = 0; jj < nxy; jj++) {
        int32_t index = (int32_t)floor(xo_random2() * size);
        index = (index == size) ? size - 1 : index;
        int32_t col = counter[index] % c->N_x, row = counter[index] / c->N_x;
        for (int n = b * (c->N_z / c->nzb); n < (b + 1) * (c->N_z / c->nzb); n++)
          if (c->mask[(((size_t)i * c->N_y + row) * c->N_x + col) * c->N_z + n] == 1) {
            xl[*u] = col;
            yl[*u] = row;
            (*u)++;
            break;
          }
        counter[index] = counter[size - 1];
        size--;
      }
    }
  free(counter);
}

/* Partition / RandomizedPartition / RandomizedSelect, XT_NHICD.c:63-126 */
static uint32_t xo_partition(xo_real *A, uint32_t p, uint32_t r) {
  xo_real x = A[r], t;
  uint32_t i = p - 1;
  for (uint32_t j = p; j < r; j++)
    if (A[j] <= x) { i++; t = A[i]; A[i] = A[j]; A[j] = t; }
  t = A[i + 1]; A[i + 1] = A[r]; A[r] = t;
  return i + 1;
}

xo_real xo_randomized_select(xo_real *A, uint32_t p, uint32_t r, uint32_t i) {
  for (;;) {
    if (p == r) return A[p];
    uint32_t rnum = (uint32_t)floor(xo_random2() * (r - p + 1));
    rnum = (rnum == r - p + 1) ? r - p : rnum;
    uint32_t j = p + rnum;
    xo_real t = A[r]; A[r] = A[j]; A[j] = t;
    uint32_t q = xo_partition(A, p, r), k = q - p + 1;
    if (i == k) return A[q];
    if (i < k) r = q - 1;
    else { p = q + 1; i = i - k; }
  }
}

/* ComputeVSC, XT_NHICD.c:128-162 */
void xo_vsc_filter(const xo_ctx *c, const xo_real *map, xo_real *out) {
  static const xo_real H[5][5] = {{0.0064, 0.0432, 0.0800, 0.0432, 0.0064},
                                  {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
                                  {0.0800, 0.5400, 1.0000, 0.5400, 0.0800},
                                  {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
                                  {0.0064, 0.0432, 0.0800, 0.0432, 0.0064}};
  for (int i = 0; i < c->N_y; i++)
    for (int j = 0; j < c->N_x; j++) {
      xo_real f = 0;
      for (int p = -2; p <= 2; p++)
        for (int q = -2; q <= 2; q++)
          if (i + p >= 0 && i + p < c->N_y && j + q >= 0 && j + q < c->N_x)
            f += H[p + 2][q + 2] * map[(size_t)(i + p) * c->N_x + (j + q)];
      out[(size_t)i * c->N_x + j] = f;
    }
}

/* VSC_based_Voxel_Line_Select, XT_NHICD.c:164-216 */
void xo_nhicd_select(xo_ctx *c, const int32_t *usn, int32_t *nsn, int32_t *xsel, int32_t *ysel) {
  int32_t nxy = c->N_x * c->N_y;
  xo_real *f = (xo_real *)malloc(sizeof(xo_real) * (size_t)nxy);
  xo_real *fc = (xo_real *)malloc(sizeof(xo_real) * (size_t)nxy);
  for (int i = 0; i < c->N_time; i++)
    for (int b = 0; b < c->nzb; b++) {
      int32_t n = (int32_t)floor(usn[i * c->nzb + b] / XO_NHICD_ITERS), idx = 0;
      xo_vsc_filter(c, &c->magmap[((size_t)i * c->nzb + b) * nxy], f);
      memcpy(fc, f, sizeof(xo_real) * (size_t)nxy);
      xo_real th = xo_randomized_select(f, 0, (uint32_t)(nxy - 1), (uint32_t)(nxy - n));
      int32_t *xl = &xsel[((size_t)i * c->nzb + b) * nxy], *yl = &ysel[((size_t)i * c->nzb + b) * nxy];
      for (int j = 0; j < c->N_y; j++)
        for (int k = 0; k < c->N_x; k++)
          if (fc[(size_t)j * c->N_x + k] > th) { xl[idx] = k; yl[idx] = j; idx++; }
      nsn[i * c->nzb + b] = idx;
    }
  free(f);
  free(fc);
}

/* update_Sinogram_Offset, XT_ICD_update.c:666-759 */
void xo_update_offset(xo_ctx *c) {
  size_t nrt = (size_t)c->N_r * c->N_t;
  xo_real *num = (xo_real *)calloc(nrt, sizeof(xo_real)), *den = (xo_real *)calloc(nrt, sizeof(xo_real));
  xo_real num_sum = 0, den_sum = 0, gamma = 0, temp, sign;
  for (int i = 0; i < c->N_r; i++)
    for (int j = 0; j < c->N_t; j++) {
      size_t o = (size_t)i * c->N_t + j;
      num[o] = 0;
      den[o] = 0;
      for (int k = 0; k < c->N_p; k++) {
        size_t s = SIDX(c, k, i, j);
        temp = (xo_real)(c->T * c->delta * sqrt(c->w[s]));
        if (c->sel[s]) {
          num[o] += c->e[s] * c->w[s];
          den[o] += c->w[s];
        } else {
          sign = (xo_real)((c->e[s] > 0) - (c->e[s] < 0));
          num[o] += temp * sign;
          den[o] = (xo_real)(den[o] + temp / fabs(c->e[s]));
        }
      }
      num_sum += c->d[o] + (num[o] / den[o]);
      den_sum = (xo_real)(den_sum + 1.0 / den[o]);
    }
  gamma = c->prm.zero_mean_offset ? num_sum / den_sum : 0;
  for (int i = 0; i < c->N_r; i++)
    for (int j = 0; j < c->N_t; j++) {
      size_t o = (size_t)i * c->N_t + j;
      c->d[o] = c->d[o] + (num[o] - gamma) / den[o];
      for (int k = 0; k < c->N_p; k++) {
        size_t s = SIDX(c, k, i, j);
        c->e[s] -= (num[o] - gamma) / den[o];
        c->sel[s] = xo_select(c, c->e[s], c->w[s]);
      }
    }
  free(num);
  free(den);
}

/* update_variance_parameter, XT_ICD_update.c:633-664 */
void xo_update_variance(xo_ctx *c) {
  size_t ns = (size_t)c->N_p * c->N_r * c->N_t;
  xo_real acc = 0, temp;
  for (size_t s = 0; s < ns; s++) {
    c->w[s] = c->w[s] * c->var_est;
    if (c->sel[s])
      temp = c->e[s] * c->e[s] * c->w[s];
    else
      temp = (xo_real)(fabs(c->e[s]) * c->delta * c->T * sqrt(c->w[s] * c->var_est));
    acc += temp;
  }
  c->var_est = acc / ((xo_real)1 * (xo_real)c->N_p * (xo_real)c->N_r * (xo_real)c->N_t);
  for (size_t s = 0; s < ns; s++) {
    c->w[s] /= c->var_est;
    c->sel[s] = xo_select(c, c->e[s], c->w[s]);
  }
}

/* updateVoxelsTimeSlices, XT_ICD_update.c:767-926 (single rank, the OpenMP
 * task loops run in their index order, which gives the same result because
 * concurrent tasks never share sinogram rows or prior neighbours). */
int xo_iterate(xo_ctx *c, int32_t iter, xo_real *avg_pct) {
  const int K = XO_NHICD_ITERS, nzb = c->nzb;
  int32_t nxy = c->N_x * c->N_y;
  long zc = 0;
  xo_real total = 0;
  xo_random_lists(c, c->usn, c->xr, c->yr);
  int32_t zstep = (int32_t)floor(c->N_z / nzb);
  for (int j = 0; j < K; j++) {
    total = 0;
    for (int half = 0; half < 2; half++) {
      for (int i = 0; i < c->N_time; i++)
        for (int b = 0; b < nzb; b += 2) {
          int idx = ((i % 2 == 0) ^ half) ? b : b + 1;
          int32_t zs = idx * zstep, ze = (idx + 1) * zstep - 1;
          ze = (idx >= nzb - 1) ? c->N_z - 1 : ze;
          int32_t u = c->usn[i * nzb + idx];
          int32_t xb = j * (int32_t)floor(u / K), xe = (j + 1) * (int32_t)floor(u / K) - 1;
          xe = (j == K - 1) ? u - 1 : xe;
          size_t lo = ((size_t)i * nzb + idx) * nxy;
          total += xo_update_voxels(c, i, zs, ze, xb, xe, &c->xr[lo], &c->yr[lo], iter, &zc,
                                    &c->magmap[lo]);
        }
      if (c->prm.update_proj_offset > 1) xo_update_offset(c);
    }
    xo_nhicd_select(c, c->usn, c->nsn, c->xn, c->yn);
    if (iter > 1 && c->prm.no_nhicd == 0) {
      for (int half = 0; half < 2; half++) {
        for (int i = 0; i < c->N_time; i++)
          for (int b = 0; b < nzb; b += 2) {
            int idx = ((i % 2 == 0) ^ half) ? b : b + 1;
            int32_t zs = idx * zstep, ze = (idx + 1) * zstep - 1;
            ze = (idx >= nzb - 1) ? c->N_z - 1 : ze;
            size_t lo = ((size_t)i * nzb + idx) * nxy;
            xo_update_voxels(c, i, zs, ze, 0, c->nsn[i * nzb + idx] - 1, &c->xn[lo], &c->yn[lo], iter,
                             &zc, &c->magmap[lo]);
          }
        if (c->prm.update_proj_offset > 1) xo_update_offset(c);
      }
    }
  }
  if (c->prm.update_var) xo_update_variance(c);
  xo_real avg = 0;
  for (int i = 0; i < c->N_time; i++)
    for (int b = 0; b < nzb; b++) {
      size_t lo = ((size_t)i * nzb + b) * nxy;
      for (int q = 0; q < c->usn[i * nzb + b]; q++)
        avg += c->magmap[lo + (size_t)c->yr[lo + q] * c->N_x + c->xr[lo + q]];
    }
  xo_real pct = 100 * avg / total;
  if (avg_pct) *avg_pct = pct;
  return pct < c->StopThreshold ? 1 : 0;
}

/* upsample_object_bilinear_2D, XT_ICD_update.c:354-386 (in and out without halo) */
void xo_upsample_xy(const xo_real *in, xo_real *out, int32_t nz, int32_t ny, int32_t nx) {
  xo_real *buf = (xo_real *)malloc(sizeof(xo_real) * (size_t)ny * 2 * nx);
  for (int s = 0; s < nz; s++) {
    const xo_real *I = &in[(size_t)s * ny * nx];
    xo_real *O = &out[(size_t)s * 4 * ny * nx];
#define IB(j, k) I[(size_t)(j) * nx + (k)]
#define BB(j, k) buf[(size_t)(j) * 2 * nx + (k)]
#define OB(j, k) O[(size_t)(j) * 2 * nx + (k)]
    for (int j = 0; j < ny; j++) {
      BB(j, 0) = IB(j, 0);
      BB(j, 1) = (xo_real)((3.0 * IB(j, 0) + IB(j, 1)) / 4.0);
      BB(j, 2 * nx - 1) = IB(j, nx - 1);
      BB(j, 2 * nx - 2) = (xo_real)((IB(j, nx - 2) + 3.0 * IB(j, nx - 1)) / 4.0);
      for (int k = 1; k < nx - 1; k++) {
        BB(j, 2 * k) = (xo_real)((IB(j, k - 1) + 3.0 * IB(j, k)) / 4.0);
        BB(j, 2 * k + 1) = (xo_real)((3.0 * IB(j, k) + IB(j, k + 1)) / 4.0);
      }
    }
    for (int k = 0; k < 2 * nx; k++) {
      OB(0, k) = BB(0, k);
      OB(1, k) = (xo_real)((3.0 * BB(0, k) + BB(1, k)) / 4.0);
      OB(2 * ny - 1, k) = BB(ny - 1, k);
      OB(2 * ny - 2, k) = (xo_real)((BB(ny - 2, k) + 3.0 * BB(ny - 1, k)) / 4.0);
    }
    for (int j = 1; j < ny - 1; j++)
      for (int k = 0; k < 2 * nx; k++) {
        OB(2 * j, k) = (xo_real)((BB(j - 1, k) + 3.0 * BB(j, k)) / 4.0);
        OB(2 * j + 1, k) = (xo_real)((3 * BB(j, k) + BB(j + 1, k)) / 4.0);
      }
#undef IB
#undef BB
#undef OB
  }
  free(buf);
}

/* upsample_object_bilinear_3D, XT_ICD_update.c:388-436 (in and out without halo) */
void xo_upsample_xyz(const xo_real *in, xo_real *out, int32_t nz, int32_t ny, int32_t nx) {
  size_t pl = (size_t)4 * ny * nx;
  xo_real *b3 = (xo_real *)malloc(sizeof(xo_real) * (size_t)nz * pl);
  xo_upsample_xy(in, b3, nz, ny, nx);
  for (size_t q = 0; q < pl; q++) {
    out[q] = b3[q];
    out[pl + q] = (xo_real)((3.0 * b3[q] + b3[pl + q]) / 4.0);
    out[(size_t)(2 * nz - 1) * pl + q] = b3[(size_t)(nz - 1) * pl + q];
    out[(size_t)(2 * nz - 2) * pl + q] = (xo_real)((3.0 * b3[(size_t)(nz - 1) * pl + q] + b3[(size_t)(nz - 2) * pl + q]) / 4.0);
  }
  for (int s = 1; s < nz - 1; s++)
    for (size_t q = 0; q < pl; q++) {
      out[(size_t)(2 * s) * pl + q] = (xo_real)((b3[(size_t)(s - 1) * pl + q] + 3.0 * b3[(size_t)s * pl + q]) / 4.0);
      out[(size_t)(2 * s + 1) * pl + q] = (xo_real)((3.0 * b3[(size_t)s * pl + q] + b3[(size_t)(s + 1) * pl + q]) / 4.0);
    }
  free(b3);
}
