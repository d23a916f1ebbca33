/*
 * ref_harness.c -- ctypes-callable wrapper around the compiled reference
 * engine (gromitsun/timbir-python Source_Code_4D_Fast), built by
 * oracle/Makefile into oracle/_ref/libxtref{32,64}.so.
 *
 * TEST INFRASTRUCTURE ONLY.  It lets the tests call the reference's own
 * routines on chosen inputs (A-matrix columns, detector response, error
 * sinogram, cost, one ICD iteration, NHICD selection, offset / variance
 * updates) so the CPU restatement in xt_oracle.c can be pinned against them.
 *
 * Set-up goes through the reference's own argsParser and initStructures, so
 * the caller passes the XT_Engine command line and must have view_info.txt in
 * the working directory (initSparseAnglesfrmFile reads it from there, and
 * argsParser opens its DEBUG log there).  The set-up that ICD_BackProject
 * does before its iteration loop (XT_ICD_update.c:952-998) is repeated here
 * in the same order.
 */
#include <getopt.h>
#include <math.h>
#include <omp.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "XT_Structures.h"
#include "XT_Constants.h"
#include "XT_AMatrix.h"
#include "XT_ICD_update.h"
#include "XT_Init.h"
#include "XT_NHICD.h"
#include "XT_Profile.h"
#include "allocate.h"
#include "randlib.h"

/* reference routines that have no prototype in the reference headers */
Real_t computeCost(Sinogram *, ScannedObject *, TomoInputs *, Real_t ***);
void initErrorSinogam(Sinogram *, ScannedObject *, TomoInputs *, Real_t **, Real_t ***);
int updateVoxelsTimeSlices(Sinogram *, ScannedObject *, TomoInputs *, Real_t **, Real_t ***, int32_t, Real_t ****, uint8_t ****);
void update_Sinogram_Offset(Sinogram *, TomoInputs *, Real_t ***);
void update_variance_parameter(Sinogram *, TomoInputs *, Real_t ***);
void upsample_object_bilinear_2D(Real_t ***, Real_t ***, int32_t, int32_t, int32_t);
void upsample_object_bilinear_3D(Real_t ***, Real_t ***, int32_t, int32_t, int32_t);
void randomly_select_x_y(ScannedObject *, TomoInputs *, uint8_t ****);

typedef struct {
  Sinogram *S;
  ScannedObject *O;
  TomoInputs *T;
  Real_t **H_r, *H_t, ***E, ****Mag;
  uint8_t ****Mask;
} xr_ctx;

xr_ctx *xr_create(int argc, char **argv) {
  xr_ctx *c = (xr_ctx *)calloc(1, sizeof(xr_ctx));
  c->S = (Sinogram *)get_spc(1, sizeof(Sinogram));
  c->O = (ScannedObject *)get_spc(1, sizeof(ScannedObject));
  c->T = (TomoInputs *)get_spc(1, sizeof(TomoInputs));
  c->T->node_num = 1;
  c->T->node_rank = 0;
  optind = 0; /* glibc: 0 re-initialises getopt, so several contexts can be made per process */
  argsParser(argc, argv, c->S, c->O, c->T);
  initStructures(c->S, c->O, c->T);
  ScannedObject *O = c->O;
  TomoInputs *T = c->T;
  Sinogram *S = c->S;
  /* The reference leaves the object (and its halo) to malloc; zero it so
   * small test volumes do not start from stale heap contents. */
  for (int i = 0; i < O->N_time; i++) memset(&O->Object[i][0][0][0], 0, sizeof(Real_t) * (size_t)(O->N_z + 2) * O->N_y * O->N_x);
  memset(&S->ProjOffset[0][0], 0, sizeof(Real_t) * (size_t)S->N_r * S->N_t);
  omp_set_num_threads(T->num_threads > 0 ? T->num_threads : 1);
  c->Mag = (Real_t ****)multialloc(sizeof(Real_t), 4, O->N_time, T->num_z_blocks, O->N_y, O->N_x);
  memset(&c->Mag[0][0][0][0], 0, sizeof(Real_t) * (size_t)O->N_time * T->num_z_blocks * O->N_y * O->N_x);
  c->Mask = (uint8_t ****)multialloc(sizeof(uint8_t), 4, O->N_time, O->N_y, O->N_x, O->N_z);
  for (int i = 0; i < O->N_time; i++)
    for (int j = 0; j < O->N_y; j++)
      for (int k = 0; k < O->N_x; k++) {
        Real_t x = O->x0 + ((Real_t)k + 0.5) * O->delta_xy;
        Real_t y = O->y0 + ((Real_t)j + 0.5) * O->delta_xy;
        uint8_t m = (x * x + y * y < T->radius_obj * T->radius_obj) ? 1 : 0;
        for (int l = 0; l < O->N_z; l++) c->Mask[i][j][k][l] = m;
      }
  c->H_r = (Real_t **)multialloc(sizeof(Real_t), 2, S->N_p, DETECTOR_RESPONSE_BINS + 1);
  c->H_t = (Real_t *)get_spc(DETECTOR_RESPONSE_BINS + 1, sizeof(Real_t));
  DetectorResponseProfile(c->H_r, c->H_t, S, O, T);
  c->E = (Real_t ***)multialloc(sizeof(Real_t), 3, S->N_p, S->N_r, S->N_t);
  memset(&c->E[0][0][0], 0, sizeof(Real_t) * (size_t)S->N_p * S->N_r * S->N_t);
  return c;
}

void xr_dims(const xr_ctx *c, int32_t *d) {
  d[0] = c->O->N_x; d[1] = c->O->N_y; d[2] = c->O->N_z; d[3] = c->O->N_time;
  d[4] = c->S->N_r; d[5] = c->S->N_t; d[6] = c->S->N_p; d[7] = c->T->num_z_blocks; d[8] = c->S->z_overlap_num;
}

void xr_derived(const xr_ctx *c, double *o) {
  o[0] = c->S->delta_r; o[1] = c->S->delta_t; o[2] = c->S->R0; o[3] = c->S->RMax; o[4] = c->O->x0; o[5] = c->O->y0;
  o[6] = c->O->delta_xy; o[7] = c->S->OffsetR; o[8] = c->T->Sigma_S_Q; o[9] = c->T->Sigma_S_Q_P;
  o[10] = c->T->Sigma_T_Q; o[11] = c->T->Sigma_T_Q_P; o[12] = c->T->Time_Filter[0];
  for (int i = 0; i < 27; i++) o[13 + i] = (&c->T->Spatial_Filter[0][0][0])[i];
}

void xr_views(const xr_ctx *c, Real_t *v, Real_t *cs, Real_t *sn, int32_t *pn, int32_t *pi) {
  int n = 0;
  for (int i = 0; i < c->S->N_p; i++) { v[i] = c->S->ViewPtr[i]; cs[i] = c->S->cosine[i]; sn[i] = c->S->sine[i]; }
  for (int t = 0; t < c->O->N_time; t++) {
    pn[t] = c->O->ProjNum[t];
    for (int k = 0; k < c->O->ProjNum[t]; k++) pi[n++] = c->O->ProjIdxPtr[t][k];
  }
}

void xr_get_hr(const xr_ctx *c, Real_t *hr) { memcpy(hr, &c->H_r[0][0], sizeof(Real_t) * (size_t)c->S->N_p * (DETECTOR_RESPONSE_BINS + 1)); }

int32_t xr_amatrix(const xr_ctx *c, int32_t row, int32_t col, int32_t view, Real_t *vals, int32_t *idx) {
  AMatrixCol a;
  Real_t v[64];
  int32_t ix[64];
  a.values = v;
  a.index = ix;
  calcAMatrixColumnforAngle(c->S, c->O, c->H_r, &a, row, col, view);
  for (int i = 0; i < a.count; i++) { vals[i] = v[i]; idx[i] = ix[i]; }
  return a.count;
}

void xr_set_sino(xr_ctx *c, const Real_t *y, const Real_t *w, const Real_t *d) {
  size_t ns = (size_t)c->S->N_p * c->S->N_r * c->S->N_t;
  memcpy(&c->S->Projection[0][0][0], y, ns * sizeof(Real_t));
  memcpy(&c->T->Weight[0][0][0], w, ns * sizeof(Real_t));
  Real_t *W = &c->T->Weight[0][0][0];
  for (size_t i = 0; i < ns; i++) W[i] /= c->T->var_est; /* computeWriteSinogram, XT_Engine.c:115-118 */
  if (d) memcpy(&c->S->ProjOffset[0][0], d, sizeof(Real_t) * (size_t)c->S->N_r * c->S->N_t);
}

void xr_set_object(xr_ctx *c, const Real_t *x) {
  size_t n = (size_t)c->O->N_z * c->O->N_y * c->O->N_x;
  for (int i = 0; i < c->O->N_time; i++) memcpy(&c->O->Object[i][1][0][0], &x[i * n], n * sizeof(Real_t));
}

void xr_get_object(const xr_ctx *c, Real_t *x) {
  size_t n = (size_t)c->O->N_z * c->O->N_y * c->O->N_x;
  for (int i = 0; i < c->O->N_time; i++) memcpy(&x[i * n], &c->O->Object[i][1][0][0], n * sizeof(Real_t));
}

void xr_get_error_sino(const xr_ctx *c, Real_t *e) { memcpy(e, &c->E[0][0][0], sizeof(Real_t) * (size_t)c->S->N_p * c->S->N_r * c->S->N_t); }
void xr_set_error_sino(xr_ctx *c, const Real_t *e) {
  size_t ns = (size_t)c->S->N_p * c->S->N_r * c->S->N_t;
  Real_t *E = &c->E[0][0][0], *W = &c->T->Weight[0][0][0];
  bool *P = &c->S->ProjSelect[0][0][0];
  memcpy(E, e, ns * sizeof(Real_t));
  for (size_t i = 0; i < ns; i++) P[i] = (fabs(E[i] * sqrt(W[i])) < c->T->ErrorSinoThresh);
}
void xr_get_weight(const xr_ctx *c, Real_t *w) { memcpy(w, &c->T->Weight[0][0][0], sizeof(Real_t) * (size_t)c->S->N_p * c->S->N_r * c->S->N_t); }
void xr_get_offset(const xr_ctx *c, Real_t *d) { memcpy(d, &c->S->ProjOffset[0][0], sizeof(Real_t) * (size_t)c->S->N_r * c->S->N_t); }
Real_t xr_get_var(const xr_ctx *c) { return c->T->var_est; }
void xr_get_magmap(const xr_ctx *c, Real_t *m) {
  memcpy(m, &c->Mag[0][0][0][0], sizeof(Real_t) * (size_t)c->O->N_time * c->T->num_z_blocks * c->O->N_y * c->O->N_x);
}
void xr_set_magmap(xr_ctx *c, const Real_t *m) {
  memcpy(&c->Mag[0][0][0][0], m, sizeof(Real_t) * (size_t)c->O->N_time * c->T->num_z_blocks * c->O->N_y * c->O->N_x);
}

void xr_init_error_sino(xr_ctx *c) { initErrorSinogam(c->S, c->O, c->T, c->H_r, c->E); }

Real_t xr_cost(xr_ctx *c, Real_t *fwd, Real_t *prior) {
  Real_t v = computeCost(c->S, c->O, c->T, c->E);
  if (fwd) *fwd = c->T->Forward_Cost;
  if (prior) *prior = c->T->Prior_Cost;
  return v;
}

int xr_iterate(xr_ctx *c, int32_t iter) {
  return updateVoxelsTimeSlices(c->S, c->O, c->T, c->H_r, c->E, iter, c->Mag, c->Mask);
}

Real_t xr_functional_substitution(const xr_ctx *c, Real_t V, Real_t th1, Real_t th2, const Real_t *nh,
                                  const Real_t *tnh, const uint8_t *fl, const uint8_t *tfl) {
  Real_t N[3][3][3], TN[2];
  bool F[3][3][3], TF[2];
  for (int i = 0; i < 27; i++) { (&N[0][0][0])[i] = nh[i]; (&F[0][0][0])[i] = fl[i] != 0; }
  for (int i = 0; i < 2; i++) { TN[i] = tnh[i]; TF[i] = tfl[i] != 0; }
  return CE_FunctionalSubstitution(V, th1, th2, c->O, c->T, N, TN, F, TF);
}

void xr_random_lists(xr_ctx *c, int32_t *usn, int32_t *xs, int32_t *ys) {
  TomoInputs *T = c->T;
  ScannedObject *O = c->O;
  size_t nxy = (size_t)O->N_x * O->N_y;
  randomly_select_x_y(O, T, c->Mask);
  for (int i = 0; i < O->N_time; i++)
    for (int b = 0; b < T->num_z_blocks; b++) {
      usn[i * T->num_z_blocks + b] = T->UpdateSelectNum[i][b];
      memcpy(&xs[(i * T->num_z_blocks + b) * nxy], T->x_rand_select[i][b], sizeof(int32_t) * nxy);
      memcpy(&ys[(i * T->num_z_blocks + b) * nxy], T->y_rand_select[i][b], sizeof(int32_t) * nxy);
    }
}

void xr_nhicd_select(xr_ctx *c, const int32_t *usn, int32_t *nsn, int32_t *xs, int32_t *ys) {
  TomoInputs *T = c->T;
  ScannedObject *O = c->O;
  size_t nxy = (size_t)O->N_x * O->N_y;
  for (int i = 0; i < O->N_time; i++)
    for (int b = 0; b < T->num_z_blocks; b++) T->UpdateSelectNum[i][b] = usn[i * T->num_z_blocks + b];
  VSC_based_Voxel_Line_Select(O, T, c->Mag);
  for (int i = 0; i < O->N_time; i++)
    for (int b = 0; b < T->num_z_blocks; b++) {
      nsn[i * T->num_z_blocks + b] = T->NHICDSelectNum[i][b];
      memcpy(&xs[(i * T->num_z_blocks + b) * nxy], T->x_NHICD_select[i][b], sizeof(int32_t) * nxy);
      memcpy(&ys[(i * T->num_z_blocks + b) * nxy], T->y_NHICD_select[i][b], sizeof(int32_t) * nxy);
    }
}

Real_t xr_randomized_select(Real_t *a, uint32_t p, uint32_t r, uint32_t i) { return RandomizedSelect(a, p, r, i); }
void xr_update_offset(xr_ctx *c) { update_Sinogram_Offset(c->S, c->T, c->E); }
void xr_update_variance(xr_ctx *c) { update_variance_parameter(c->S, c->T, c->E); }
void xr_srandom2(uint32_t s) { srandom2(s); }
double xr_random2(void) { return random2(); }

void xr_upsample_xy(const Real_t *in, Real_t *out, int32_t nz, int32_t ny, int32_t nx) {
  Real_t ***I = (Real_t ***)multialloc(sizeof(Real_t), 3, nz, ny, nx);
  Real_t ***O = (Real_t ***)multialloc(sizeof(Real_t), 3, nz + 2, 2 * ny, 2 * nx);
  memcpy(&I[0][0][0], in, sizeof(Real_t) * (size_t)nz * ny * nx);
  upsample_object_bilinear_2D(O, I, nz, ny, nx);
  memcpy(out, &O[1][0][0], sizeof(Real_t) * (size_t)nz * 4 * ny * nx);
  multifree(I, 3);
  multifree(O, 3);
}

void xr_upsample_xyz(const Real_t *in, Real_t *out, int32_t nz, int32_t ny, int32_t nx) {
  Real_t ***I = (Real_t ***)multialloc(sizeof(Real_t), 3, nz, ny, nx);
  Real_t ***O = (Real_t ***)multialloc(sizeof(Real_t), 3, 2 * nz + 2, 2 * ny, 2 * nx);
  memcpy(&I[0][0][0], in, sizeof(Real_t) * (size_t)nz * ny * nx);
  upsample_object_bilinear_3D(O, I, nz, ny, nx);
  memcpy(out, &O[1][0][0], sizeof(Real_t) * (size_t)2 * nz * 4 * ny * nx);
  multifree(I, 3);
  multifree(O, 3);
}

void xr_destroy(xr_ctx *c) {
  if (!c) return;
  fclose(c->T->debug_file_ptr);
  multifree(c->E, 3);
  multifree(c->H_r, 2);
  free(c->H_t);
  multifree(c->Mask, 4);
  multifree(c->Mag, 4);
  free(c);
}
