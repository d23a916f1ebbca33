/*
 * xt_gen.h -- C ABI of libxtgen.so: seeded synthetic inputs for the engine.
 *
 * The reference ships no datasets (its beamline HDF5 files and phantoms are
 * external), so benchmarks and tests use seeded synthetic stand-ins written
 * in the reference's own input formats:
 *   view_info.txt        "<time> - <angle_deg>," per view
 *                        (4D_Recon_Launcher_for_Real_Data/XT_MBIR_Reconstruction.py:7-13)
 *   projection_n0.bin    float32 [N_p][N_r][N_t], y = ln(I0 / counts)
 *   weight_n0.bin        float32 [N_p][N_r][N_t], w = counts
 *                        (4D_Recon_Launcher_for_Real_Data/XT_Projections.py:28-123)
 * The forward model is the reference's own A (calcAMatrixColumnforAngle)
 * summed in the reference's order, so a noiseless sinogram equals the
 * reference's initErrorSinogam projection bit for bit.
 */
#ifndef XT_GEN_H
#define XT_GEN_H
#include <stddef.h>
#include <stdint.h>

#include "xt_geom.h"

#ifdef __cplusplus
extern "C" {
#endif

/* angle_i = i * 180 / n_p degrees, time_i = i (uniform views over [0, 180)). */
int xtgen_views_uniform(int32_t n_p, double *times, double *angles_deg);
/* TIMBIR interlaced views, gen_interlaced_views_0_to_Inf
 * (4D_Recon_Launcher_for_Real_Data/XT_Interlaced_Angles.py:107-139):
 * K sub-frames per rotation of N_theta angles, bit-reversed sub-frame offsets,
 * time_i = view index / K, angle in degrees (unwrapped, >= 0). */
int xtgen_views_interlaced(int32_t K, int32_t N_theta, int32_t n_p, double *times, double *angles_deg);
/* Writes view_info.txt and rounds the arrays to the values a reader parses. */
int xtgen_write_view_file(const char *path, int32_t n, double *times, double *angles_deg);

typedef struct {
  int32_t n_ellipsoids; /* random ellipsoids */
  double mu_max;        /* attenuation of each ellipsoid ~ U(0, mu_max) per voxel length */
  int32_t n_moving;     /* the first n_moving ellipsoids translate over frames */
  double max_shift;     /* voxels per frame */
  int32_t growing;      /* add one ellipsoid that grows over frames */
  uint64_t seed;
} xtgen_phantom_spec;

/* x: float [N_time][N_z][N_y][N_x] */
int xtgen_phantom(const xtgen_phantom_spec *spec, int32_t N_time, int32_t N_z, int32_t N_y, int32_t N_x, float *x);

/* A x on the host (reference A, reference summation order, OpenMP over views).
 * x: [N_time][N_z][N_y][N_x]; ax: [N_p][N_r][N_t]. */
int xtgen_forward(const xt_params *prm, const double *times, const double *angles_deg, int32_t n, const float *x,
                  float *ax);

/* counts ~ Poisson(I0 exp(-ax)) (at least 1), y = ln(I0/counts), w = counts;
 * then a zinger_frac fraction of entries gets y += U(zinger_lo, zinger_hi).
 * Deterministic for a seed, independent of the thread count. */
int xtgen_measure(size_t n, const float *ax, double I0, double zinger_frac, double zinger_lo, double zinger_hi,
                  uint64_t seed, float *y, float *w);

int xtgen_write_bin(const char *path, const float *a, size_t n, int as_double);

/* The engine's host-side set-up without a GPU: derived geometry, view tables
 * (cos, sin, frame of each view) and H_r[N_p][65], exactly as libxtgpu
 * uploads them.  Any output may be NULL.  Returns 0 or -1 (message in err). */
int xtgen_geometry(const xt_params *prm, const double *times, const double *angles_deg, int32_t n, xt_geom *g,
                   float *cosv, float *sinv, int32_t *frame_of_view, float *hr, char *err, size_t errlen);
/* calcAMatrixColumnforAngle on the host for one (row, col, view). */
int32_t xtgen_amatrix(const xt_params *prm, const double *times, const double *angles_deg, int32_t n, int32_t row,
                      int32_t col, int32_t view, float *vals, int32_t *idx);

#ifdef __cplusplus
}
#endif
#endif
