/*
 * xtg.h -- C ABI of libxtgpu.so, the B200 TIMBIR/MBIR reconstruction core.
 *
 * The reference engine (gromitsun/timbir-python Source_Code_4D_Fast) is one C
 * program whose hot path is ICD_BackProject and the routines under it.  This
 * library replaces those routines; the host program XT_Engine (same command
 * line, same files) calls it through the entry points below.  Each entry
 * point names the reference routine it replaces.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Host arrays are row-major float32 in the
 *     reference's layouts:
 *       sinogram arrays (projection y, weight w, error e)  [N_p][N_r][N_t]
 *       projection offset d                                [N_r][N_t]
 *       object x                                           [N_time][N_z][N_y][N_x]
 *       magnitude-update map                               [N_time][nzb][N_y][N_x]
 *   - Every call returns 0 or a negative XTG_E* status; xtg_last_error()
 *     gives the message.  No exception crosses the ABI.  A context is not
 *     thread safe; use one context per host thread.
 *   - All device state lives in one context on the current CUDA device; the
 *     library never falls back to the CPU: without a usable sm_100 GPU,
 *     xtg_create fails with XTG_E_CUDA.
 */
#ifndef XTG_H
#define XTG_H
#include <stddef.h>
#include <stdint.h>

#include "xt_geom.h"

#ifdef __cplusplus
extern "C" {
#endif

#define XTG_ABI_VERSION 1

enum {
  XTG_OK = 0,
  XTG_E_ARG = -1,     /* bad argument or configuration */
  XTG_E_CUDA = -2,    /* CUDA runtime error (no device, out of memory, launch failure) */
  XTG_E_STATE = -3,   /* call out of order (e.g. iterate before the sinogram is uploaded) */
  XTG_E_NUMERIC = -4, /* non-finite value met in an update (theta2 <= 0 with zero prior weight) */
  XTG_E_TIMEOUT = -5  /* a bounded device-side wait gave up */
};

/* A-matrix storage used by the ICD kernel.
 *   XTG_A_FP32:    entries computed in the kernel at every column visit,
 *                  bit-identical to calcAMatrixColumnforAngle
 *                  (XT_AMatrix.c:50-110); no extra memory.
 *   XTG_A_TABLE32: the same FP32 entries precomputed once per context into
 *                  an HBM column table (4 B offset + 4 B value per entry).
 *   XTG_A_FP16:    the column table with FP16 values and one FP32 scale per
 *                  (frame, column) -- the FP16-A precision form.
 *   XTG_A_AUTO:    xtg_set_options picks TABLE32 when the table fits in free
 *                  device memory with 2 GiB to spare, else FP16, else FP32. */
enum { XTG_A_FP32 = 0, XTG_A_FP16 = 1, XTG_A_TABLE32 = 2, XTG_A_AUTO = 3 };

/* Update order.
 *   XTG_ORDER_PARALLEL: many columns in flight at once (the B200 schedule);
 *   XTG_ORDER_SEQUENTIAL: one column at a time, slices in increasing z, in
 *       the list order given -- the reference's own order, for parity tests. */
enum { XTG_ORDER_PARALLEL = 0, XTG_ORDER_SEQUENTIAL = 1 };

typedef struct xtg_ctx xtg_ctx;

/* Per-iteration statistics, the quantities updateVoxelsTimeSlices logs and
 * tests (XT_ICD_update.c:884-925). */
typedef struct {
  double avg_update_pct;   /* 100 * sum(MagUpdateMap over the random lists) / vox_mag */
  double mag_sum;          /* sum of MagUpdateMap over the random lists */
  double vox_mag;          /* sum |x| over voxels updated in the last chunk's random pass */
  double total_pix;        /* voxels in the random lists */
  int64_t voxel_updates;   /* voxel updates performed (random + NHICD), zero-skipped excluded */
  int64_t zero_skipped;    /* voxels skipped by ZERO_SKIPPING */
  int64_t columns;         /* column (z-line) work items processed */
  int32_t converged;       /* avg_update_pct < voxel_thresh */
  float ms;                /* device time of the iteration, CUDA events */
} xtg_stats;

/* Replaces argsParser/initStructures/DetectorResponseProfile set-up
 * (XT_Init.c:277-629, XT_Profile.c:128-217, XT_ICD_update.c:952-978).
 * view_times / view_angles_deg: the n entries of view_info.txt. */
int xtg_create(const xt_params *prm, const double *view_times, const double *view_angles_deg, int32_t n,
               xtg_ctx **out);
void xtg_destroy(xtg_ctx *ctx);
const char *xtg_last_error(void);
int xtg_abi_version(void);

/* dims[11]: N_x, N_y, N_z, N_time, N_r, N_t, N_p, nzb, zovl, amax, and the
 * number of x-y columns inside the reconstruction disk (radius_obj) */
int xtg_dims(const xtg_ctx *ctx, int32_t *dims);
/* Geometry and tables exactly as the GPU uses them (host copies). */
int xtg_geometry(const xtg_ctx *ctx, xt_geom *g);
int xtg_get_hr(const xtg_ctx *ctx, float *hr /*[N_p][65]*/);

/* Options: A storage, update order, concurrent columns (0 = device default),
 * seed of the GPU visiting order. */
int xtg_set_options(xtg_ctx *ctx, int32_t a_mode, int32_t order, int32_t max_columns, uint64_t seed);
/* Forward projector.  Both give the same values (bit-identical in FP32, the
 * reference's summation order; FP64 sums otherwise):
 *   XTG_PROJ_AUTO:   at the first projection the context builds a bin-major
 *                    A table (rows (view, bin), entries in the reference's
 *                    (row, column) order; 8 B per entry) when it fits in free
 *                    device memory next to the ICD column table and 2 GiB to
 *                    spare, and projects from it; else as XTG_PROJ_GATHER.
 *   XTG_PROJ_GATHER: A evaluated on the fly for each (view, 32 bins), no
 *                    table.
 * xtg_get_projector reports XTG_PROJ_TABLE once the table is in use (or
 * XTG_PROJ_GATHER; XTG_PROJ_AUTO before the first projection) and its entry
 * count.  No reference counterpart (B200 layout choices). */
enum { XTG_PROJ_AUTO = 0, XTG_PROJ_GATHER = 1, XTG_PROJ_TABLE = 2 };
int xtg_set_projector(xtg_ctx *ctx, int32_t kind);
int xtg_get_projector(const xtg_ctx *ctx, int32_t *in_use, int64_t *table_entries);
/* The options in force (XTG_A_AUTO resolved to the storage it picked);
 * outputs may be NULL.  No reference counterpart. */
int xtg_get_options(const xtg_ctx *ctx, int32_t *a_mode, int32_t *order, int32_t *max_columns, uint64_t *seed);
/* Parallel schedule: z slices per ICD work piece (0 = chosen from the L2 size,
 * the default).  Each column visit is cut into pieces of at most this many
 * slices, visited piece-major, so the error-sinogram and weight rows in
 * flight fit in L2.  The sequential order always takes whole items.  No
 * reference counterpart (a B200 scheduling knob). */
int xtg_set_zslab(xtg_ctx *ctx, int32_t slices);
/* The z slices per work piece the parallel schedule uses now. */
int xtg_get_zslab(const xtg_ctx *ctx, int32_t *slices);

/* One z slab of a volume split over processes, one GPU each -- the
 * reference's MPI ranks (XT_Init.c:290-294: a rank owns N_z / ranks slices
 * and the matching N_t / ranks detector rows, Length_T / ranks).  Create the
 * context with those N_t and length_t, then give it device planes
 * [N_time][N_y][N_x] (caller-owned) for each side that has a neighbour:
 * send_* receive this slab's boundary slice (slice 0 below, slice N_z - 1
 * above), recv_* hold the neighbour's adjacent slice.  At the start of every
 * xtg_icd_iteration and after each of its ICD launches (the reference
 * exchanges after every half-pass, XT_ICD_update.c:816-880) the library
 * fills send_*, drains its stream and calls exchange(user, phase); the hook
 * moves the planes between processes (NCCL, MPI, ...) and returns 0 once
 * recv_* hold the neighbours' slices.  The ICD updates then see those slices
 * as z neighbours (XT_VoxUpdate.c:94-99), and the MAP cost's prior includes
 * the pairs into the slab above (XT_ICD_update.c:203-205); summing the
 * slabs' xtg_map_cost_fp64 and xtg_stats over processes gives the whole
 * volume's cost and stop statistic.  NULL planes: no neighbour on that side.
 * Variance and offset re-estimation are refused for slabs (they need sums
 * over every slab inside the iteration). */
typedef int (*xtg_exchange_fn)(void *user, int32_t phase);
int xtg_set_slab(xtg_ctx *ctx, float *send_below, float *send_above, const float *recv_below, const float *recv_above,
                 xtg_exchange_fn exchange, void *user);
/* One exchange now (after the object changed outside xtg_icd_iteration, e.g.
 * a warm start or an upload, and before a MAP cost); every slab of the volume
 * must make the call. */
int xtg_slab_exchange(xtg_ctx *ctx);

/* genSinogram_fromBin + computeWriteSinogram (XT_genSinogram.c:264-300,
 * XT_Engine.c:89-121): y, w and the offset d (NULL = zero).  Weights are
 * divided by the variance estimate on the device, like the reference. */
int xtg_upload_sino(xtg_ctx *ctx, const float *y, const float *w, const float *d);
/* xtg_upload_sino followed by xtg_init_error_sino for the object on the
 * device (e = y - Ax - d, bit-identical), with the host-to-device copies of
 * y, w and d on a second stream while Ax is projected.  Host buffers in
 * pinned memory let the copies overlap.  No XT_Engine counterpart (the
 * reference reads the sinogram and initialises e as two steps, XT_Engine.c
 * computeWriteSinogram and XT_ICD_update.c initErrorSinogam). */
int xtg_upload_sino_start(xtg_ctx *ctx, const float *y, const float *w, const float *d);
/* Counts ingest, genSinogram_subsampleCounts (XT_genSinogram.c:303-374):
 * bright [N_r*mult_xy][N_t*mult_z] and weight counts [N_p][N_r*mult_xy][N_t*mult_z]
 * are binned to y = log(bright/counts) (+ BH_QUAD_COEF * y^2) and w = counts. */
int xtg_upload_counts(xtg_ctx *ctx, const float *bright, const float *counts, double bh_quad_coef,
                      const float *d);
int xtg_upload_object(xtg_ctx *ctx, const float *x);
int xtg_download_object(xtg_ctx *ctx, float *x);
/* xtg_download_object without blocking the host: the object is copied to a
 * staging buffer of the library at once (later calls may change it), and
 * from there to x on a second stream, overlapping the work queued next (a
 * pinned x makes the copy asynchronous).  x is complete after
 * xtg_download_wait, which blocks until the last such copy has arrived; do
 * not read or reuse x before it.  A second start waits on the device for the
 * first copy to leave the staging buffer.  No XT_Engine counterpart. */
int xtg_download_object_start(xtg_ctx *ctx, float *x);
int xtg_download_wait(xtg_ctx *ctx);
int xtg_get_error_sino(xtg_ctx *ctx, float *e);
int xtg_set_error_sino(xtg_ctx *ctx, const float *e);
int xtg_get_weight(xtg_ctx *ctx, float *w);
int xtg_get_offset(xtg_ctx *ctx, float *d);
int xtg_set_offset(xtg_ctx *ctx, const float *d);
int xtg_get_magmap(xtg_ctx *ctx, float *m);
int xtg_set_magmap(xtg_ctx *ctx, const float *m);
int xtg_get_variance(xtg_ctx *ctx, double *var_est);
int xtg_set_variance(xtg_ctx *ctx, double var_est);

/* A-matrix column generation on the GPU, calcAMatrixColumnforAngle
 * (XT_AMatrix.c:50-110), for n (row, col, view) triples.  vals/idx hold amax
 * slots per triple, cnt the entry count. */
int xtg_amatrix(xtg_ctx *ctx, int32_t n, const int32_t *rows, const int32_t *cols, const int32_t *views,
                float *vals, int32_t *idx, int32_t *cnt);
/* Forward projection A x of the current object, FP32, every sinogram entry
 * summed over columns in the reference's (row, column) order, so the result
 * is bit-identical to the reference's (initErrorSinogam + forward_project_voxel_AMat1D,
 * XT_ICD_update.c:551-569, XT_ForwardProject.c:8-25).  ax may be NULL
 * (result stays on the device). */
int xtg_forward_project(xtg_ctx *ctx, float *ax);
/* e = y - A x - d in FP32 (initErrorSinogam, XT_ICD_update.c:538-597), with
 * the reference's projector, which leaves out the delta_t factor the voxel
 * update applies to A (XT_ForwardProject.c:17 against XT_VoxUpdate.c:27,67):
 * with delta_t != 1 only a zero object gives the e the update assumes, in
 * the reference as here.  The starts this library computes itself (FBP,
 * multi-resolution, learned) set e = y - A delta_t x - d instead. */
int xtg_init_error_sino(xtg_ctx *ctx);
/* Warm start: object := filtered backprojection of y - d (ramp filter and
 * linearly interpolated backprojection over each frame's views; 0 outside
 * the reconstruction disk, clamped at 0 with positivity), then
 * e = y - Ax - d.  No XT_Engine counterpart: the reference starts from zero
 * or a coarser stage (initObject, XT_ICD_update.c:443-536), and its
 * launchers compute FBP outside the engine (XT_FBP_Reconstruction.py). */
int xtg_init_object_fbp(xtg_ctx *ctx);
/* Device-to-device object transfer in the engine's device layout
 * [N_time][N_y][N_x][N_z] (z fastest; the channels-last volume layout of
 * xtg_cnn.h with nb = N_time).  xtg_object_from_device zeroes columns outside
 * the reconstruction disk and clamps at 0 with positivity; e is not updated
 * (call xtg_init_error_sino).  No reference counterpart. */
int xtg_object_to_device(xtg_ctx *ctx, float *dst);
int xtg_object_from_device(xtg_ctx *ctx, const float *src);

/* upsample_object_bilinear_2D / _3D (XT_ICD_update.c:354-436) on the GPU:
 * in [nt][nz][ny][nx] (host) -> out [nt][2nz or nz][2ny][2nx] (host), bit for
 * bit the reference's values (the initICD 2 / 3 starts of XT_Engine). */
int xtg_upsample(xtg_ctx *ctx, const float *in, float *out, int32_t nt, int32_t nz, int32_t ny, int32_t nx,
                 int32_t with_z);

/* Multi-resolution start, the launcher's coarse-to-fine stages in one call:
 * reconstruct the same data on a grid with voxels twice as large in x-y (and
 * z with XTG_MULTIRES_Z), from its FBP image, for coarse_iters ICD
 * iterations; then object := that reconstruction upsampled as above (0
 * outside the disk, clamped with positivity) and e = y - Ax - d.  With
 * XTG_MULTIRES_BIN the coarse grid sees a detector binned 2x in bins (and
 * rows with XTG_MULTIRES_Z): weights summed, projections weight-averaged --
 * the binning genSinogram_subsampleCounts (XT_genSinogram.c:303-374) applies
 * to counts -- four times fewer sinogram entries per coarse iteration.  The
 * coarse context is kept for later calls with the same flags.  No XT_Engine
 * counterpart (the launcher runs the stages as separate XT_Engine processes
 * with --initICD 2/3). */
enum { XTG_MULTIRES_Z = 1, XTG_MULTIRES_BIN = 2 };
int xtg_init_object_multires(xtg_ctx *ctx, int32_t coarse_iters, int32_t flags);
/* e = y - A delta_t x - d with FP64 accumulation, rounded to FP32: the
 * periodic resync that removes the drift of incremental FP32 updates.  A
 * delta_t is the matrix the voxel update subtracts (XT_VoxUpdate.c:27,67), so
 * this is the error sinogram the reference carries from its zero start.  The
 * same pass yields the MAP cost of the current object in FP64 (outputs may be
 * NULL). */
int xtg_resync_fp64(xtg_ctx *ctx, double *cost, double *forward, double *prior);
/* MAP cost of the current object (computeCost, XT_ICD_update.c:181-314),
 * evaluated in FP64 from e64 = y - A delta_t x - d (not from the running e). */
int xtg_map_cost_fp64(xtg_ctx *ctx, double *cost, double *forward, double *prior);
/* MAP cost from the running error sinogram in FP64 arithmetic. */
int xtg_map_cost_running(xtg_ctx *ctx, double *cost, double *forward, double *prior);

/* Zinger weight refresh: ProjSelect = |e sqrt(w)| < T for every sinogram
 * entry (XT_ICD_update.c:576-580, 659-663, 750-753; XT_VoxUpdate.c:76-79).
 * sel (may be NULL) receives the mask; nsel the count of selected entries. */
int xtg_zinger_refresh(xtg_ctx *ctx, uint8_t *sel, int64_t *nsel);

/* One reference iteration, updateVoxelsTimeSlices (XT_ICD_update.c:767-926):
 * a random visiting order cut in 10 chunks, each chunk followed by NHICD
 * selection and (iter > 1, NHICD on) an NHICD pass; offset and variance
 * updates when enabled.  Voxels of a column's z-line are updated together. */
int xtg_icd_iteration(xtg_ctx *ctx, int32_t iter, xtg_stats *st);

/* Column update over an explicit work list (the hot kernel alone):
 * items[4*q] = {frame, row, col, block}, block = -1 for the whole z-line.
 * Used by the sequential parity tests and the benchmark. */
int xtg_update_columns(xtg_ctx *ctx, int32_t iter, int32_t n_items, const int32_t *items, xtg_stats *st);

/* NHICD selection, VSC_based_Voxel_Line_Select + ComputeVSC
 * (XT_NHICD.c:128-216): 5x5 Hamming filter of the magnitude-update map, the
 * order statistic at N_xy - floor(update_select_num/10), the columns above it.
 * update_select_num[N_time*nzb] in; nhicd_num[N_time*nzb] and, when not
 * NULL, the lists (x, y) [N_time][nzb][N_xy] out (raster order). */
int xtg_nhicd_select(xtg_ctx *ctx, const int32_t *update_select_num, int32_t *nhicd_num, int32_t *x_sel,
                     int32_t *y_sel, float *thresholds);

/* update_Sinogram_Offset (XT_ICD_update.c:666-759) and
 * update_variance_parameter (XT_ICD_update.c:633-664). */
int xtg_update_offset(xtg_ctx *ctx);
int xtg_update_variance(xtg_ctx *ctx);

/* NHICD thresholds without allocating any device memory.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc -- hosts
 * that own every device buffer through their own pool and allow no
 * allocation once started (for instance a beamline acquisition loop, where
 * cudaMalloc's implicit device-wide synchronisation would stall the detector
 * stream).  The caller passes device buffers: magmap [nmaps][ny][nx] (the
 * magnitude-update maps), thresholds [nmaps] (out: for map s the kth[s]-th
 * smallest value, 1-based, of its 5x5 Hamming-filtered map, as
 * xtg_nhicd_select computes) and, when not NULL, select [nmaps][ny][nx] (out:
 * 1 where the filtered value exceeds the threshold); kth is a host array.
 * Work is queued on `stream` (a cudaStream_t, NULL = default stream) and is
 * complete when that stream is.
 * Scratch is one fixed array inside the library, XTG_NOALLOC_MAX_ELEMS floats
 * (4 MiB) plus XTG_NOALLOC_MAX_MAPS ints, held on every GPU that loads the
 * library until the process exits; larger inputs are rejected with XTG_E_ARG.
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other host threads) race on it and must be serialised by the caller.
 * The resolved address is kept for the life of the process: after a
 * cudaDeviceReset of a device, do not call this entry point on that device
 * again.  A CUDA error already pending when it is called (from the caller's
 * own earlier work) is reported as XTG_E_CUDA and left pending. */
#define XTG_NOALLOC_MAX_ELEMS (1 << 20)
#define XTG_NOALLOC_MAX_MAPS 256
int xtg_nhicd_threshold_noalloc(const float *magmap, int32_t nmaps, int32_t ny, int32_t nx, const int32_t *kth,
                                float *thresholds, uint8_t *select, void *stream);

/* Device bytes held by the context. */
int64_t xtg_device_bytes(const xtg_ctx *ctx);
/* Kernel launches issued by this context since creation (all kernels). */
int64_t xtg_launch_count(const xtg_ctx *ctx);
/* Device time (ms) of the ICD column kernel in the last xtg_icd_iteration /
 * xtg_update_columns call, the random-pass column work items it processed and
 * the number of ICD kernel launches it issued. */
int xtg_last_kernel_time(const xtg_ctx *ctx, float *ms, int64_t *items, int64_t *launches);

#ifdef __cplusplus
}
#endif
#endif
