/*
 * xt_gen.c -- seeded synthetic phantoms and sinograms (libxtgen.so).
 *
 * Stand-ins for the reference's external datasets, written in its input
 * formats (see include/xt_gen.h).  Everything is deterministic for a seed:
 * each sinogram entry draws from its own counter-based stream, so results do
 * not depend on the OpenMP thread count.
 */
#include "../../include/xt_gen.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* splitmix64 (Steele, Lea, Flood 2014) */
static inline uint64_t sm64(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline double u01(uint64_t *s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

int xtgen_views_uniform(int32_t n_p, double *times, double *angles) {
  if (n_p <= 0) return -1;
  for (int32_t i = 0; i < n_p; i++) {
    times[i] = (double)i;
    angles[i] = (double)i * 180.0 / (double)n_p;
  }
  return 0;
}

static uint32_t bitrev(uint32_t v, int bits) {
  uint32_t r = 0;
  for (int b = 0; b < bits; b++) r |= ((v >> b) & 1u) << (bits - 1 - b);
  return r;
}

int xtgen_views_interlaced(int32_t K, int32_t N_theta, int32_t n_p, double *times, double *angles) {
  if (K <= 0 || N_theta <= 0 || n_p <= 0 || N_theta % K != 0 || (K & (K - 1)) != 0) return -1;
  const int32_t L = N_theta / K;
  int bits = 0;
  while ((1 << bits) < K) bits++;
  const double dtheta = 180.0 / (double)N_theta;
  for (int32_t i = 0; i < n_p; i++) {
    const double v = (double)i * K + (double)bitrev((uint32_t)((i / L) % K), bits);
    times[i] = v / K;
    angles[i] = v * dtheta;
  }
  return 0;
}

int xtgen_write_view_file(const char *path, int32_t n, double *times, double *angles) {
  FILE *fp = fopen(path, "w");
  if (!fp) return -1;
  char a[64], b[64];
  for (int32_t i = 0; i < n; i++) {
    /* fixed notation: the reader treats '-' and '+' as separators */
    snprintf(a, sizeof(a), "%.12f", times[i]);
    snprintf(b, sizeof(b), "%.12f", angles[i]);
    fprintf(fp, "%s - %s,\n", a, b);
    times[i] = atof(a);
    angles[i] = atof(b);
  }
  return fclose(fp) == 0 ? 0 : -1;
}

int xtgen_phantom(const xtgen_phantom_spec *s, int32_t nt, int32_t nz, int32_t ny, int32_t nx, float *x) {
  if (!s || nt <= 0 || nz <= 0 || ny <= 0 || nx <= 0) return -1;
  const int ne = s->n_ellipsoids + (s->growing ? 1 : 0);
  double *P = (double *)calloc((size_t)(ne > 0 ? ne : 1) * 10, sizeof(double));
  uint64_t st = s->seed ^ 0xA5A5A5A5DEADBEEFULL;
  const double R = 0.5 * (nx < ny ? nx : ny);
  for (int e = 0; e < ne; e++) {
    double *q = &P[e * 10];
    const double rad = 0.6 * R * sqrt(u01(&st)), th = 2.0 * M_PI * u01(&st);
    q[0] = 0.5 * nx + rad * cos(th);                 /* centre x (voxels) */
    q[1] = 0.5 * ny + rad * sin(th);                 /* centre y */
    q[2] = nz * (0.3 + 0.4 * u01(&st));              /* centre z */
    q[3] = R * (0.08 + 0.30 * u01(&st));             /* semi-axis a */
    q[4] = R * (0.08 + 0.30 * u01(&st));             /* semi-axis b */
    q[5] = nz * (0.25 + 0.5 * u01(&st)) + 1.0;       /* semi-axis c */
    q[6] = M_PI * u01(&st);                          /* rotation about z */
    q[7] = s->mu_max * u01(&st);                     /* attenuation */
    const double vth = 2.0 * M_PI * u01(&st);
    const int moving = e < s->n_moving;
    q[8] = moving ? s->max_shift * u01(&st) * cos(vth) : 0.0; /* velocity, voxels/frame */
    q[9] = moving ? s->max_shift * u01(&st) * sin(vth) : 0.0;
    if (s->growing && e == ne - 1) { q[3] *= 0.5; q[4] *= 0.5; q[5] *= 0.5; }
  }
  const size_t plane = (size_t)ny * nx;
#pragma omp parallel for schedule(static)
  for (int64_t fz = 0; fz < (int64_t)nt * nz; fz++) {
    const int f = (int)(fz / nz), z = (int)(fz % nz);
    float *o = &x[(size_t)fz * plane];
    memset(o, 0, plane * sizeof(float));
    for (int e = 0; e < ne; e++) {
      const double *q = &P[e * 10];
      double g = 1.0;
      if (s->growing && e == ne - 1) g = 1.0 + (double)f / (double)nt;
      const double cx = q[0] + q[8] * f, cy = q[1] + q[9] * f, cz = q[2];
      const double a = q[3] * g, b = q[4] * g, c = q[5] * g, cs = cos(q[6]), sn = sin(q[6]);
      const double dz = ((z + 0.5) - cz) / c;
      if (dz * dz >= 1.0) continue;
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nx; k++) {
          const double dx = (k + 0.5) - cx, dy = (j + 0.5) - cy;
          const double u = (dx * cs + dy * sn) / a, v = (-dx * sn + dy * cs) / b;
          if (u * u + v * v + dz * dz < 1.0) o[(size_t)j * nx + k] += (float)q[7];
        }
    }
  }
  free(P);
  return 0;
}

int xtgen_forward(const xt_params *prm, const double *times, const double *angles, int32_t n, const float *x,
                  float *ax) {
  xt_geom g;
  xt_views v;
  char err[512];
  if (xt_geom_derive(prm, &g, err, sizeof(err)) != 0) {
    fprintf(stderr, "%s\n", err);
    return -1;
  }
  if (xt_views_build(&g, times, angles, n, &v, err, sizeof(err)) != 0) {
    fprintf(stderr, "%s\n", err);
    return -1;
  }
  float *hr = (float *)malloc(sizeof(float) * (size_t)g.N_p * XT_HR_STRIDE);
  xt_detector_response(&g, &v, hr);
  const size_t plane = (size_t)g.N_y * g.N_x;
  /* z-lines contiguous: xt[f][j][k][z] */
  float *xt = (float *)malloc(sizeof(float) * (size_t)g.N_time * plane * g.N_z);
  for (int f = 0; f < g.N_time; f++)
    for (int z = 0; z < g.N_z; z++)
      for (size_t q = 0; q < plane; q++)
        xt[((size_t)f * plane + q) * g.N_z + z] = x[((size_t)f * g.N_z + z) * plane + q];
  const size_t per_view = (size_t)g.N_r * g.N_t;
  memset(ax, 0, sizeof(float) * per_view * g.N_p);
  /* each view is owned by one thread; per entry the sum runs over columns in
   * (row, col) order, the order of the reference's initErrorSinogam */
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < g.N_p; p++) {
    const int f = v.frame_of_view[p];
    float vals[XT_AMAX];
    int32_t idx[XT_AMAX];
    float *o = &ax[(size_t)p * per_view];
    for (int j = 0; j < g.N_y; j++)
      for (int k = 0; k < g.N_x; k++) {
        const int32_t cnt = xt_amatrix_host(&g, &v, hr, j, k, p, vals, idx);
        const float *xl = &xt[((size_t)f * plane + (size_t)j * g.N_x + k) * g.N_z];
        for (int m = 0; m < cnt; m++) {
          float *row = &o[(size_t)idx[m] * g.N_t];
          const float a = vals[m];
          for (int z = 0; z < g.N_z; z++) {
            const float pix = xl[z];
            for (int r = 0; r < g.zovl; r++) row[z * g.zovl + r] += pix * a;
          }
        }
      }
  }
  free(xt);
  free(hr);
  xt_views_free(&v);
  return 0;
}

/* Poisson(lam): inversion for small lam, PTRS (Hormann 1993, "The transformed
 * rejection method for generating Poisson random variables") otherwise. */
static double poisson(uint64_t *s, double lam) {
  if (lam <= 0) return 0;
  if (lam < 10.0) {
    const double L = exp(-lam);
    double p = 1.0, k = -1.0;
    do {
      k += 1.0;
      p *= u01(s);
    } while (p > L && k < 1000.0);
    return k;
  }
  const double slam = sqrt(lam), loglam = log(lam);
  const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
  const double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
  for (;;) {
    const double U = u01(s) - 0.5, V = u01(s), us = 0.5 - fabs(U);
    const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
    if (us >= 0.07 && V <= vr) return k;
    if (k < 0 || (us < 0.013 && V > us)) continue;
    if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return k;
  }
}

int xtgen_measure(size_t n, const float *ax, double I0, double zfrac, double zlo, double zhi, uint64_t seed,
                  float *y, float *w) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t s = seed * 0xD1B54A32D192ED03ULL ^ ((uint64_t)i * 0x9E3779B97F4A7C15ULL);
    sm64(&s);
    double cnt = poisson(&s, I0 * exp(-(double)ax[i]));
    if (cnt < 1.0) cnt = 1.0;
    double yy = log(I0 / cnt);
    if (zfrac > 0 && u01(&s) < zfrac) yy += zlo + (zhi - zlo) * u01(&s);
    y[i] = (float)yy;
    w[i] = (float)cnt;
  }
  return 0;
}

int xtgen_geometry(const xt_params *prm, const double *times, const double *angles, int32_t n, xt_geom *g,
                   float *cosv, float *sinv, int32_t *fov, float *hr, char *err, size_t errlen) {
  xt_geom G;
  xt_views v;
  if (xt_geom_derive(prm, &G, err, errlen) != 0) return -1;
  if (xt_views_build(&G, times, angles, n, &v, err, errlen) != 0) return -1;
  if (g) *g = G;
  if (cosv) memcpy(cosv, v.cosv, sizeof(float) * (size_t)n);
  if (sinv) memcpy(sinv, v.sinv, sizeof(float) * (size_t)n);
  if (fov) memcpy(fov, v.frame_of_view, sizeof(int32_t) * (size_t)n);
  if (hr) xt_detector_response(&G, &v, hr);
  xt_views_free(&v);
  return 0;
}

int32_t xtgen_amatrix(const xt_params *prm, const double *times, const double *angles, int32_t n, int32_t row,
                      int32_t col, int32_t view, float *vals, int32_t *idx) {
  xt_geom G;
  xt_views v;
  char err[256];
  if (xt_geom_derive(prm, &G, err, sizeof(err)) != 0) return -1;
  if (xt_views_build(&G, times, angles, n, &v, err, sizeof(err)) != 0) return -1;
  float *hr = (float *)malloc(sizeof(float) * (size_t)G.N_p * XT_HR_STRIDE);
  xt_detector_response(&G, &v, hr);
  const int32_t c = xt_amatrix_host(&G, &v, hr, row, col, view, vals, idx);
  free(hr);
  xt_views_free(&v);
  return c;
}

int xtgen_write_bin(const char *path, const float *a, size_t n, int as_double) {
  FILE *fp = fopen(path, "wb");
  if (!fp) return -1;
  size_t wr;
  if (as_double) {
    double *d = (double *)malloc(n * sizeof(double));
    for (size_t i = 0; i < n; i++) d[i] = a[i];
    wr = fwrite(d, sizeof(double), n, fp);
    free(d);
  } else {
    wr = fwrite(a, sizeof(float), n, fp);
  }
  return (fclose(fp) == 0 && wr == n) ? 0 : -1;
}
