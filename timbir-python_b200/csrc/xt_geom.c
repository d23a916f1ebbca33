/*
 * xt_geom.c -- host-side geometry of the TIMBIR engine.
 *
 * Rounding convention: the reference is C99 on Real_t = float; an expression
 * that mixes a float with a double literal or a libm call is evaluated in
 * double and rounded to float on assignment.  The helpers here spell that out
 * with explicit casts, so the tables handed to the GPU (cos/sin, H_r, filter,
 * geometry scalars) hold the reference's float values bit for bit.
 */
#include "xt_geom.h"

#include <ctype.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define XT_PI 3.14159265358979323846
#define XT_PI_2 1.57079632679489661923132169163975144
#define XT_PI_4 0.785398163397448309615660845819875721

void xt_params_default(xt_params *p) {
  /* argsParser defaults (XT_Init.c:513-531); the reference zero-fills the rest */
  memset(p, 0, sizeof(*p));
  p->cost_thresh = 100;
  p->Est_of_Var = 1;
}

static double xt_dist(int a, int b, int c, int d) { /* distance2node, XT_Init.c:204 */
  return (float)sqrt(pow((float)a - 1.0, 2.0) + pow((float)b - 1.0, 2.0) + pow((float)c - 1.0, 2.0) +
                     pow((float)d - 1.0, 2.0));
}

int xt_geom_derive(const xt_params *p, xt_geom *g, char *err, size_t errlen) {
  memset(g, 0, sizeof(*g));
  /* HU conversion of sigma_s / sigma_t (XT_Init.c:510-511, 543, 546) */
  float slope = (float)((1000 - 0) / (0.521225397034623 * 1.0 - 0.496372335005353 * 0.001205) / 0.0001);
  float chu = (float)(-slope * (0.496372335005353 * 0.001205 * 0.0001));
  float sigma_s = (float)(p->sigma_s - chu) / slope;
  float sigma_t = (float)(p->sigma_t - chu) / slope;
  float mult_xy = (float)p->delta_xy, mult_z = (float)p->delta_z;
  float length_r = (float)p->length_r, length_t = (float)p->length_t;
  float rot = (float)p->rotation_center;
  g->MRF_P = (float)p->p;
  g->C_S = (float)p->c_s;
  g->C_T = (float)p->c_t;
  g->alpha = (float)p->alpha;
  g->T = (float)p->zingerT;
  g->delta = (float)p->zingerDel;
  g->var_est = (float)p->Est_of_Var;
  g->StopThreshold = (float)p->voxel_thresh;
  g->radius_obj = (float)p->radius_obj;
  g->Rtime0 = (float)p->Rtime0;
  g->delta_Rtime = (float)p->Rtime_delta;
  g->mult_xy = mult_xy;
  g->mult_z = mult_z;
  g->N_r = p->N_r;
  g->N_p = p->num_projections;
  g->N_time = p->Rtime_num;
  g->N_t = p->N_t;
  if (p->sinobin == 3) {
    /* counts ingest works on detector bins binned by mult_xy x mult_z (XT_Init.c:608-616) */
    g->N_t = (int32_t)(g->N_t / mult_z);
    g->N_r = (int32_t)(g->N_r / mult_xy);
    rot /= mult_xy;
  }
  float dxy_mult = (p->sinobin == 3) ? 1.0f : mult_xy;
  float dz_mult = (p->sinobin == 3) ? 1.0f : mult_z;
  g->zovl = (int32_t)dz_mult;
  if (g->N_r <= 0 || g->N_t <= 0 || g->N_p <= 0 || g->N_time <= 0) {
    snprintf(err, errlen, "ERROR: N_r, N_t, num_projections and Rtime_num must be positive");
    return -1;
  }
  if ((int32_t)dz_mult <= 0 || (int32_t)dxy_mult <= 0) {
    snprintf(err, errlen, "ERROR: delta_xy and delta_z must be at least 1");
    return -1;
  }
  if (g->N_t % (int32_t)dz_mult != 0) {
    snprintf(err, errlen, "ERROR: initStructures: Cannot do reconstruction since delta_z = %d does not divide %d",
             (int32_t)dz_mult, g->N_t);
    return -1;
  }
  if (g->N_r % (int32_t)dxy_mult != 0) {
    snprintf(err, errlen, "ERROR: initStructures: Cannot do reconstruction since delta_xy = %d does not divide %d",
             (int32_t)dxy_mult, g->N_r);
    return -1;
  }
  g->delta_r = length_r / (g->N_r);
  g->delta_t = length_t / (g->N_t);
  g->R0 = -rot * g->delta_r;
  g->RMax = (g->N_r - rot) * g->delta_r;
  g->T0 = (float)(-length_t / 2.0);
  g->N_x = (int32_t)(g->N_r / dxy_mult);
  g->N_y = g->N_x;
  g->N_z = (int32_t)(g->N_t / dz_mult);
  g->delta_xy = dxy_mult * g->delta_r;
  g->delta_z = dz_mult * g->delta_t;
  g->x0 = g->R0;
  g->y0 = (float)(-length_r / 2.0);
  g->OffsetR = (float)((g->delta_xy / sqrt(2.0) + g->delta_r / 2.0) / XT_HR_BINS);
  g->Sigma_S_Q = (float)pow((sigma_s * mult_xy), 2.0);
  g->Sigma_S_Q_P = (float)pow(sigma_s * mult_xy, 2.0 - g->MRF_P);
  g->Sigma_T_Q = (float)pow((sigma_t * g->delta_Rtime), 2.0);
  g->Sigma_T_Q_P = (float)pow(sigma_t * g->delta_Rtime, 2.0 - g->MRF_P);
  g->nzb = (int32_t)(2 * floor(p->num_threads / g->N_time));
  if (g->nzb < 2)
    g->nzb = 2;
  else if (g->nzb > g->N_z)
    g->nzb = g->N_z;
  if (g->nzb % 2 != 0) {
    /* the reference's even/odd block schedule indexes block nzb for odd nzb
     * (XT_ICD_update.c:803, 826); refuse instead of reading past the lists */
    snprintf(err, errlen, "ERROR: number of z blocks (%d) must be even; choose num_threads so that 2*floor(num_threads/Rtime_num) <= N_z is even", g->nzb);
    return -1;
  }
  g->zstep = (int32_t)floor(g->N_z / g->nzb);
  g->amax = (int32_t)ceil(3 * g->delta_xy / g->delta_r);
  if (g->amax > XT_AMAX) {
    snprintf(err, errlen, "ERROR: delta_xy/delta_r too large (%d A-matrix entries per view, at most %d)", g->amax, XT_AMAX);
    return -1;
  }
  /* prior weights, initFilter (XT_Init.c:210-256) */
  float prior_const = mult_xy * mult_xy * mult_xy * g->delta_Rtime;
  float sum = 0;
  g->TF = (float)(1.0 / xt_dist(0, 1, 1, 1));
  sum = (float)(sum + 2.0 * g->TF);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        int q = (i * 3 + j) * 3 + k;
        if (q != 13) {
          float t1 = (float)(1.0 / xt_dist(1, i, j, k));
          g->SF[q] = t1;
          sum = sum + t1;
        } else {
          g->SF[q] = 0;
        }
      }
  for (int q = 0; q < 27; q++) g->SF[q] = prior_const * g->SF[q] / sum;
  g->TF = prior_const * g->TF / sum;
  return 0;
}

int xt_views_build(const xt_geom *g, const double *times, const double *angles_deg, int32_t n, xt_views *v,
                   char *err, size_t errlen) {
  memset(v, 0, sizeof(*v));
  if (n != g->N_p) {
    snprintf(err, errlen, "ERROR: Number of projections read is %d and expected is %d", n, g->N_p);
    return -1;
  }
  v->N_p = n;
  v->N_time = g->N_time;
  v->angle = (float *)calloc(n, sizeof(float));
  v->time = (float *)calloc(n, sizeof(float));
  v->cosv = (float *)calloc(n, sizeof(float));
  v->sinv = (float *)calloc(n, sizeof(float));
  v->view_start = (int32_t *)calloc(g->N_time, sizeof(int32_t));
  v->view_num = (int32_t *)calloc(g->N_time, sizeof(int32_t));
  v->view_idx = (int32_t *)calloc(n, sizeof(int32_t));
  v->frame_of_view = (int32_t *)calloc(n, sizeof(int32_t));
  for (int32_t i = 0; i < n; i++) {
    v->angle[i] = (float)((float)angles_deg[i] * XT_PI / 180.0);
    v->time[i] = (float)times[i];
    v->cosv[i] = (float)cos(v->angle[i]);
    v->sinv[i] = (float)sin(v->angle[i]);
  }
  /* views to reconstruction frames, initSparseAnglesOfObject (XT_Init.c:98-125):
   * views are taken in file order; a frame closes when a view's time reaches
   * the frame's end time, and the last frame takes everything left. */
  int32_t frame = 0, num = 0, start = 0;
  float t2 = g->Rtime0 + g->delta_Rtime;
  for (int32_t i = 0; i < n; i++) {
    while (v->time[i] >= t2 && frame + 1 < g->N_time) {
      v->view_start[frame] = start;
      v->view_num[frame] = num;
      start += num;
      t2 += g->delta_Rtime;
      frame++;
      num = 0;
    }
    v->view_idx[start + num] = i;
    v->frame_of_view[i] = frame;
    num++;
  }
  v->view_start[frame] = start;
  v->view_num[frame] = num;
  return 0;
}

void xt_views_free(xt_views *v) {
  free(v->angle); free(v->time); free(v->cosv); free(v->sinv);
  free(v->view_start); free(v->view_num); free(v->view_idx); free(v->frame_of_view);
  memset(v, 0, sizeof(*v));
}

/* view_info.txt parser (XT_Init.c:56-75, 130-162).  White space, newlines
 * included, is skipped; a token is a run of alphanumerics and '.'; the
 * character that ends it decides its meaning: '-' makes it the time of the
 * following views, ',' makes it an angle in degrees, anything else is a
 * format error.  End of file ends the scan and drops an unterminated token. */
int32_t xt_read_view_file(const char *path, double **times, double **angles, char *err, size_t errlen) {
  FILE *fp = fopen(path, "r");
  if (!fp) {
    snprintf(err, errlen, "ERROR: Error in reading file %s", path);
    return -1;
  }
  size_t cap = 1024, n = 0;
  double *t = (double *)malloc(cap * sizeof(double)), *a = (double *)malloc(cap * sizeof(double));
  char tok[128];
  size_t tl = 0;
  double cur_time = 0;
  int ch;
  while ((ch = fgetc(fp)) != EOF) {
    if (isspace(ch)) continue;
    if (isalnum(ch) || ch == '.') {
      if (tl + 1 < sizeof(tok)) tok[tl++] = (char)ch;
      continue;
    }
    tok[tl] = '\0';
    if (ch == '-') {
      cur_time = (float)atof(tok);
    } else if (ch == ',') {
      if (tl > 0) {
        if (n == cap) {
          cap *= 2;
          t = (double *)realloc(t, cap * sizeof(double));
          a = (double *)realloc(a, cap * sizeof(double));
        }
        t[n] = cur_time;
        a[n] = atof(tok);
        n++;
      }
    } else {
      snprintf(err, errlen, "ERROR: initSparseAnglesfrmFile: File %s is not correctly formatted to be read", path);
      fclose(fp);
      free(t);
      free(a);
      return -2;
    }
    tl = 0;
  }
  fclose(fp);
  *times = t;
  *angles = a;
  return (int32_t)n;
}

void xt_detector_response(const xt_geom *g, const xt_views *v, float *hr) {
  float *vp = (float *)malloc(sizeof(float) * XT_PROFILE_RES);
  float beam[XT_BEAM_RES], bsum = 0;
  /* Hamming beam profile normalised to unit area, XT_Profile.c:107-123 */
  for (int i = 0; i < XT_BEAM_RES; i++) {
    beam[i] = (float)(0.54 - 0.46 * cos((2 * XT_PI / XT_BEAM_RES) * i));
    bsum = bsum + beam[i];
  }
  for (int i = 0; i < XT_BEAM_RES; i++) beam[i] /= bsum;
  float r0 = -(g->delta_r) / 2, step = (g->delta_r) / XT_BEAM_RES;
  float tconst = (XT_PROFILE_RES) / (2 * g->delta_xy);
  for (int k = 0; k < v->N_p; k++) {
    /* trapezoidal voxel line-integral profile of view k, XT_Profile.c:46-103 */
    float ang = v->angle[k], maxv;
    while (ang > XT_PI_2) ang = (float)(ang - XT_PI_2);
    while (ang < 0) ang = (float)(ang + XT_PI_2);
    maxv = (ang <= XT_PI_4) ? (float)(g->delta_xy / cos(ang)) : (float)(g->delta_xy / cos(XT_PI_2 - ang));
    float c4 = (float)cos(XT_PI_4);
    float d1 = (float)(c4 * cos((XT_PI_4 - ang))), d2 = (float)(c4 * fabs((cos((XT_PI_4 + ang)))));
    float LC = 1 - d1, LN = 1 - d2, RN = 1 + d2, RC = 1 + d1;
    for (int j = 0; j < XT_PROFILE_RES; j++) {
      float t = (float)(2.0 * j / XT_PROFILE_RES);
      if (t <= LC || t >= RC)
        vp[j] = 0;
      else if (t > RN)
        vp[j] = maxv * (RC - t) / (RC - RN);
      else if (t >= LN)
        vp[j] = maxv;
      else
        vp[j] = maxv * (t - LC) / (LN - LC);
    }
    /* profile convolved with the beam, sampled at 64 offsets, XT_Profile.c:150-171 */
    for (int i = 0; i < XT_HR_BINS; i++) {
      float rmin = i * g->OffsetR - g->delta_xy, s = 0;
      for (int q = 0; q < XT_BEAM_RES; q++) {
        float r = r0 + q * step;
        int32_t pi = (int32_t)floor((r - rmin) * tconst);
        if (pi >= 0 && pi <= XT_PROFILE_RES - 1) s += (vp[pi] * beam[q]);
      }
      hr[(size_t)k * XT_HR_STRIDE + i] = s;
    }
    hr[(size_t)k * XT_HR_STRIDE + XT_HR_BINS] = 0.0f;
  }
  free(vp);
}

int32_t xt_amatrix_host(const xt_geom *g, const xt_views *v, const float *hr, int32_t row, int32_t col, int32_t p,
                        float *vals, int32_t *idx) {
  float x = (float)(g->x0 + ((float)col + 0.5) * g->delta_xy);
  float y = (float)(g->y0 + ((float)row + 0.5) * g->delta_xy);
  float r = x * v->cosv[p] - y * v->sinv[p];
  float rmin = r - g->delta_xy, rmax = r + g->delta_xy;
  if (rmax < g->R0 || rmin > g->RMax) return 0;
  int32_t imin = (int32_t)floor((rmin - g->R0) / g->delta_r);
  int32_t imax = (int32_t)floor((rmax - g->R0) / g->delta_r);
  if (imax >= g->N_r) imax = g->N_r - 1;
  if (imin < 0) imin = 0;
  const float *H = &hr[(size_t)p * XT_HR_STRIDE];
  int32_t n = 0;
  for (int32_t j = imin; j <= imax; j++) {
    float rc = (float)(g->R0 + (((float)j) + 0.5) * g->delta_r);
    float dr = fabsf(r - rc);
    int32_t id = (int32_t)floor(dr / g->OffsetR);
    if (id >= 0 && id < XT_HR_BINS) {
      float w1 = dr - id * g->OffsetR, w2 = g->OffsetR - w1;
      float f1 = (w2 * H[id] + w1 * H[id + 1]) / g->OffsetR;
      if (f1 > 0) {
        vals[n] = f1;
        idx[n] = j;
        n++;
      }
    }
  }
  return n;
}

int xt_in_mask(const xt_geom *g, int32_t j, int32_t k) {
  float x = (float)(g->x0 + ((float)k + 0.5) * g->delta_xy);
  float y = (float)(g->y0 + ((float)j + 0.5) * g->delta_xy);
  return (x * x + y * y < g->radius_obj * g->radius_obj) ? 1 : 0;
}
