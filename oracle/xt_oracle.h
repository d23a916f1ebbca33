/*
 * xt_oracle.h -- CPU restatement of the reference TIMBIR engine's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker.  The product (libxtgpu.so, XT_Engine) never links it.
 *
 * Every function restates one reference function of
 * gromitsun/timbir-python Source_Code_4D_Fast (cited per function in
 * xt_oracle.c), keeping the reference's float/double promotion order so that
 * the FP32 build reproduces the compiled reference bit for bit.  The oracle is
 * pinned against the compiled reference (oracle/_ref, built by
 * oracle/Makefile) and against the golden fixtures in tests/golden.
 *
 * Built twice: libxtoracle32.so (xo_real = float, like the default reference
 * build) and libxtoracle64.so (xo_real = double, like -DREAL_IS_DOUBLE).
 *
 * Array layouts are the reference's, flattened row-major:
 *   sinogram arrays  [N_p][N_r][N_t]        (t fastest)
 *   offset           [N_r][N_t]
 *   object           [N_time][N_z][N_y][N_x] (no halo on the API; x fastest)
 *   mag update map   [N_time][num_z_blocks][N_y][N_x]
 */
#ifndef XT_ORACLE_H
#define XT_ORACLE_H
#include <stdint.h>

#ifdef XO_DOUBLE
typedef double xo_real;
#else
typedef float xo_real;
#endif

/* Command-line level parameters, as argsParser (XT_Init.c:452-629) stores
 * them after atof()/atoi().  sigma_s / sigma_t are the raw CLI values (HU-like);
 * the HU conversion of XT_Init.c:510-511,543,546 is applied inside. */
typedef struct {
  double p, sigma_s, sigma_t, c_s, c_t;
  double mult_xy, mult_z, length_r, length_t, rot_center, alpha;
  double Rtime0, Rtime_delta, zingerT, zingerDel, var_est;
  double voxel_thresh, radius_obj;
  int32_t N_r, N_t, N_p, N_time, num_threads;
  int32_t positivity;          /* -DPOSITIVITY_CONSTRAINT */
  int32_t no_nhicd;            /* --no_NHICD */
  int32_t update_proj_offset;  /* --updateProjOffset */
  int32_t zero_mean_offset;    /* --EnforceZeroMeanOffset */
  int32_t update_var;          /* --do_VarEst */
} xo_params;

typedef struct xo_ctx xo_ctx;

/* dims[] order returned by xo_dims */
enum { XO_NX, XO_NY, XO_NZ, XO_NTIME, XO_NR, XO_NT, XO_NP, XO_NZB, XO_ZOVL, XO_NDIMS };

xo_ctx *xo_create(const xo_params *prm, const double *view_times, const double *view_angles_deg);
void xo_destroy(xo_ctx *c);
void xo_dims(const xo_ctx *c, int32_t *dims);

/* Scalars derived by initStructures / initFilter (XT_Init.c:277-448, :210-256):
 * out[0..] = delta_r, delta_t, R0, RMax, x0, y0, delta_xy, OffsetR,
 *            Sigma_S_Q, Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P, Time_Filter,
 *            Spatial_Filter[27] (i,j,k order) */
void xo_derived(const xo_ctx *c, double *out);
void xo_views(const xo_ctx *c, xo_real *view_rad, xo_real *cosv, xo_real *sinv,
              int32_t *proj_num /*[N_time]*/, int32_t *proj_idx /*[N_p], frame-major*/);
void xo_get_hr(const xo_ctx *c, xo_real *hr /*[N_p][65]*/);
int32_t xo_amatrix(const xo_ctx *c, int32_t row, int32_t col, int32_t view,
                   xo_real *vals, int32_t *idx);

void xo_set_sino(xo_ctx *c, const xo_real *y, const xo_real *w, const xo_real *d);
void xo_set_object(xo_ctx *c, const xo_real *x);
void xo_get_object(const xo_ctx *c, xo_real *x);
void xo_get_error_sino(const xo_ctx *c, xo_real *e);
void xo_set_error_sino(xo_ctx *c, const xo_real *e);
void xo_get_offset(const xo_ctx *c, xo_real *d);
void xo_get_weight(const xo_ctx *c, xo_real *w);
void xo_get_magmap(const xo_ctx *c, xo_real *m);
void xo_set_magmap(xo_ctx *c, const xo_real *m);
xo_real xo_get_var(const xo_ctx *c);

void xo_forward_project(const xo_ctx *c, xo_real *ax /*[N_p][N_r][N_t]*/);
void xo_init_error_sino(xo_ctx *c);
/* e = y - delta_t A x - d (the voxel update's matrix; see xt_oracle.c) */
void xo_init_error_sino_model(xo_ctx *c);
/* z slab of a volume split over ranks (see xt_oracle.c) */
void xo_set_slab(xo_ctx *c, int32_t below, int32_t above);
void xo_get_boundary(const xo_ctx *c, xo_real *lo, xo_real *hi);
void xo_set_halo(xo_ctx *c, const xo_real *lo, const xo_real *hi);
/* MAP cost of the object with FP64 sums (see xt_oracle.c) */
double xo_map_cost_fp64(const xo_ctx *c, double *fwd, double *prior);
xo_real xo_cost(xo_ctx *c, xo_real *forward, xo_real *prior);

xo_real xo_functional_substitution(const xo_ctx *c, xo_real V, xo_real th1, xo_real th2,
                                   const xo_real *nhood /*27*/, const xo_real *tnhood /*2*/,
                                   const uint8_t *flags /*27*/, const uint8_t *tflags /*2*/);

/* One reference iteration (updateVoxelsTimeSlices).  Returns the stop flag,
 * writes the stop statistic. */
int xo_iterate(xo_ctx *c, int32_t iter, xo_real *avg_update_percentage);

/* NHICD selection (VSC_based_Voxel_Line_Select) on the current map with the
 * given per-(frame,block) update counts; returns list sizes and lists. */
void xo_nhicd_select(xo_ctx *c, const int32_t *update_select_num,
                     int32_t *nhicd_num, int32_t *x_sel, int32_t *y_sel);
void xo_vsc_filter(const xo_ctx *c, const xo_real *map /*[N_y][N_x]*/, xo_real *out);
xo_real xo_randomized_select(xo_real *a, uint32_t p, uint32_t r, uint32_t i);
void xo_random_lists(xo_ctx *c, int32_t *update_select_num, int32_t *x_sel, int32_t *y_sel);

void xo_update_offset(xo_ctx *c);
void xo_update_variance(xo_ctx *c);

void xo_srandom2(uint32_t seed);
double xo_random2(void);

void xo_upsample_xy(const xo_real *in, xo_real *out, int32_t nz, int32_t ny, int32_t nx);
void xo_upsample_xyz(const xo_real *in, xo_real *out, int32_t nz, int32_t ny, int32_t nx);

#endif
