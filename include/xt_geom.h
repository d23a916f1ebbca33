/*
 * xt_geom.h -- host-side geometry of the TIMBIR engine (C99).
 *
 * The command-line parameters of XT_Engine, the geometry and prior constants
 * derived from them, the view/time tables and the detector-response table.
 * Derivations follow the reference engine's argsParser / initStructures
 * (Source_Code_4D_Fast/XT_Init.c:277-448, :452-629), keeping its float/double
 * rounding so the GPU kernels see the exact values the reference computes.
 */
#ifndef XT_GEOM_H
#define XT_GEOM_H
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XT_HR_BINS 64        /* DETECTOR_RESPONSE_BINS */
#define XT_HR_STRIDE 65      /* H_r row length: 64 bins + a trailing zero */
#define XT_PROFILE_RES 1536  /* PROFILE_RESOLUTION */
#define XT_BEAM_RES 512      /* BEAM_RESOLUTION */
#define XT_NHICD_CHUNKS 10   /* NHICD_Iterations, XT_Init.c:438 */
#define XT_AMAX 12           /* largest A-matrix entry count per (column, view) supported */

/* The XT_Engine command line, after atof()/atoi() (XT_Init.c:457-589).  The
 * two flags at the end are this engine's runtime forms of the reference's
 * compile-time macros POSITIVITY_CONSTRAINT and REAL_IS_DOUBLE. */
typedef struct {
  double p, sigma_s, sigma_t, c_s, c_t, delta_xy, delta_z, length_r, length_t;
  double voxel_thresh, cost_thresh, rotation_center, alpha, Rtime0, Rtime_delta;
  double radius_obj, zingerT, zingerDel, Est_of_Var;
  int32_t iter, sinobin, initICD, writeTiff, Rtime_num, num_projections, N_r, N_t;
  int32_t detector_slice_begin, detector_slice_num, num_threads, phantom_N_xy, phantom_N_z;
  int32_t updateProjOffset, x_start, x_width;
  int32_t EnforceZeroMeanOffset, time_reg, RMSE_converged, WritePerIter, no_NHICD;
  int32_t only_Edge_Updates, initMagUpMap, do_VarEst, dont_reconstruct, readSino4mHDF, NoNoise;
  int32_t positivity, real_is_double;
} xt_params;

/* Derived geometry (all float values rounded exactly as the reference's float
 * build rounds them). */
typedef struct {
  int32_t N_r, N_t, N_p, N_x, N_y, N_z, N_time, zovl, nzb, zstep, amax;
  float delta_r, delta_t, R0, RMax, T0, x0, y0, delta_xy, delta_z, OffsetR;
  float mult_xy, mult_z;
  float MRF_P, C_S, C_T, alpha, Sigma_S_Q, Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P;
  float SF[27]; /* spatial filter, [dz][dy][dx] of the 3x3x3 neighbourhood */
  float TF;     /* temporal filter */
  float T, delta, var_est, StopThreshold, radius_obj, Rtime0, delta_Rtime;
} xt_geom;

/* View tables.  Views of frame i are view_idx[view_start[i] .. +view_num[i]). */
typedef struct {
  int32_t N_p, N_time;
  float *angle, *time, *cosv, *sinv;
  int32_t *view_start, *view_num, *view_idx, *frame_of_view;
} xt_views;

void xt_params_default(xt_params *p);
/* 0 on success, negative with a message in err on a configuration error
 * (the reference's exit(1) paths, XT_Init.c:302-310). */
int xt_geom_derive(const xt_params *p, xt_geom *g, char *err, size_t errlen);
int xt_views_build(const xt_geom *g, const double *times, const double *angles_deg, int32_t n, xt_views *v,
                   char *err, size_t errlen);
void xt_views_free(xt_views *v);
/* Parses view_info.txt ("time - angle," entries, XT_Init.c:56-75, 130-162).
 * Returns the entry count or a negative value; arrays are malloc'd. */
int32_t xt_read_view_file(const char *path, double **times, double **angles_deg, char *err, size_t errlen);
/* H_r[N_p][65] (XT_Profile.c:46-171). */
void xt_detector_response(const xt_geom *g, const xt_views *v, float *hr);
/* calcAMatrixColumnforAngle (XT_AMatrix.c:50-110) on the host; returns the count. */
int32_t xt_amatrix_host(const xt_geom *g, const xt_views *v, const float *hr, int32_t row, int32_t col, int32_t view,
                        float *vals, int32_t *idx);
/* Column (j,k) inside the object-support disk (XT_ICD_update.c:958-974). */
int xt_in_mask(const xt_geom *g, int32_t j, int32_t k);

#ifdef __cplusplus
}
#endif
#endif
