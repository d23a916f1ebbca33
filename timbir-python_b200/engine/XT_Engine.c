/*
 * XT_Engine.c -- drop-in replacement of the reference's XT_Engine program on
 * one B200.
 *
 * Same command line (xt_cli.c), same input files in the working directory,
 * same output files and layouts, same exit codes as the reference program
 * (Source_Code_4D_Fast/XT_Engine.c:128-172 main, XT_ICD_update.c:928-1094
 * ICD_BackProject); the reconstruction itself runs in libxtgpu.so through the
 * C ABI of include/xtg.h.  One process drives one GPU: the reference's MPI
 * z-slab ranks are replaced by one device-resident volume, so file names use
 * rank 0 (the "_n0" suffix) as a single-rank reference run does.
 *
 * Inputs:  view_info.txt, projection_n0.bin + weight_n0.bin (--sinobin 1) or
 *          bright_n0.bin + weight_n0.bin (--sinobin 3), proj_offset_n0.bin
 *          (--updateProjOffset 1|3), object_n0_time_<i>.bin and
 *          variance_estimate_n0.bin (--initICD 1|2|3), mag_update_map_n0.bin
 *          (--initMagUpMap).
 * Outputs: object_n0_time_<i>.bin, proj_offset_n0.bin, variance_estimate_n0.bin,
 *          mag_update_map_n0.bin, cost_n0.bin, DEBUG_n0_delta_xy_<a>_delta_z_<b>.log.
 * Element type of every .bin file: float32, or float64 with --real_is_double
 * (the reference's -DREAL_IS_DOUBLE build).
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "xt_cli.h"
#include "xtg.h"
#include "xtg_cnn.h"

static FILE *g_log = NULL;
static int g_dbl = 0;

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void logf_(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
static void logf_(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  if (g_log) {
    vfprintf(g_log, fmt, ap);
    fflush(g_log);
  }
  va_end(ap);
}

/* Read4mBin (XT_IOMisc.c:79-96): a missing file is fatal (exit status 1, as
 * in the reference); a short read is logged with the reference's message and
 * the run continues, the unread rest of the array left at zero (the
 * reference continues with whatever its buffer held there). */
static int read_bin(const char *name, float *dst, size_t n) {
  char file[512];
  snprintf(file, sizeof(file), "%s.bin", name);
  FILE *fp = fopen(file, "rb");
  if (!fp) {
    logf_("ERROR: error in reading file %s\n", file);
    fprintf(stderr, "ERROR: error in reading file %s\n", file);
    return -1;
  }
  size_t got;
  if (g_dbl) {
    double *t = (double *)malloc(n * sizeof(double));
    if (!t) {
      fclose(fp);
      logf_("ERROR: out of host memory reading %s\n", file);
      return -1;
    }
    got = fread(t, sizeof(double), n, fp);
    for (size_t i = 0; i < got; i++) dst[i] = (float)t[i];
    free(t);
  } else {
    got = fread(dst, sizeof(float), n, fp);
  }
  fclose(fp);
  if (got != n) {
    logf_("ERROR: Number of elements read does not match required, required = %zu, read = %zu\n", n, got);
    fprintf(stderr, "WARNING: %s: read %zu of %zu elements; the rest is taken as zero\n", file, got, n);
    memset(dst + got, 0, (n - got) * sizeof(float));
  }
  return 0;
}

/* Write2Bin / Append2Bin (XT_IOMisc.c:58-77) */
static int write_bin(const char *name, const float *src, size_t n, const char *mode) {
  char file[512];
  snprintf(file, sizeof(file), "%s.bin", name);
  FILE *fp = fopen(file, mode);
  if (!fp) {
    logf_("ERROR: Write2Bin: Cannot open file %s\n", file);
    return -1;
  }
  size_t put;
  if (g_dbl) {
    double *t = (double *)malloc(n * sizeof(double));
    for (size_t i = 0; i < n; i++) t[i] = src[i];
    put = fwrite(t, sizeof(double), n, fp);
    free(t);
  } else {
    put = fwrite(src, sizeof(float), n, fp);
  }
  return (fclose(fp) == 0 && put == n) ? 0 : -1;
}

static int write_scalar(const char *name, double v, const char *mode) {
  float f = (float)v;
  if (g_dbl) {
    char file[512];
    snprintf(file, sizeof(file), "%s.bin", name);
    FILE *fp = fopen(file, mode);
    if (!fp) return -1;
    size_t put = fwrite(&v, sizeof(double), 1, fp);
    return (fclose(fp) == 0 && put == 1) ? 0 : -1;
  }
  return write_bin(name, &f, 1, mode);
}

static int write_outputs(xtg_ctx *ctx, const int32_t *dims) {
  const int N_x = dims[0], N_y = dims[1], N_z = dims[2], N_time = dims[3], N_r = dims[4], N_t = dims[5];
  const size_t vol = (size_t)N_z * N_y * N_x;
  float *x = (float *)malloc(sizeof(float) * vol * N_time);
  float *d = (float *)malloc(sizeof(float) * (size_t)N_r * N_t);
  if (xtg_download_object(ctx, x) || xtg_get_offset(ctx, d)) {
    logf_("ERROR: %s\n", xtg_last_error());
    free(x);
    free(d);
    return -1;
  }
  char name[256];
  int rc = 0;
  /* write_ObjectProjOff2TiffBinPerIter, XT_IOMisc.c:224-254 */
  for (int i = 0; i < N_time; i++) {
    snprintf(name, sizeof(name), "object_n0_time_%d", i);
    rc |= write_bin(name, x + (size_t)i * vol, vol, "wb");
  }
  rc |= write_bin("proj_offset_n0", d, (size_t)N_r * N_t, "wb");
  free(x);
  free(d);
  return rc;
}

/* The sinogram and the offset d (genSinogram_fromBin / _subsampleCounts,
 * XT_genSinogram.c:264-374; the offset of XT_Init.c:340-366, replicated from
 * the coarser stage's detector with initICD 2 / 3 and counts ingest). */
static int load_sinogram(xtg_ctx *ctx, const xt_params *P, const int32_t *dims) {
  const int N_r = dims[4], N_t = dims[5], N_p = dims[6];
  const size_t ns = (size_t)N_p * N_r * N_t, nrt = (size_t)N_r * N_t;
  float *d = NULL, *t = NULL, *y = NULL, *w = NULL;
  int rc = -1;
  if (P->updateProjOffset == 1 || P->updateProjOffset == 3) {
    d = (float *)calloc(nrt, sizeof(float));
    if (!d) goto out;
    int pxy = 1, pz = 1;
    if (P->initICD == 3) pxy = pz = 2;
    if (P->initICD == 2) pxy = 2;
    if (P->sinobin == 3 && (pxy > 1 || pz > 1)) {
      t = (float *)calloc((size_t)(N_r / pxy) * (N_t / pz), sizeof(float));
      if (!t || read_bin("proj_offset_n0", t, (size_t)(N_r / pxy) * (N_t / pz))) goto out;
      for (int i = 0; i < N_r / pxy; i++)
        for (int j = 0; j < N_t / pz; j++)
          for (int a = 0; a < pxy; a++)
            for (int b = 0; b < pz; b++) d[(size_t)(i * pxy + a) * N_t + j * pz + b] = t[(size_t)i * (N_t / pz) + j];
    } else if (read_bin("proj_offset_n0", d, nrt)) {
      goto out;
    }
  }
  if (P->sinobin == 1) {
    y = (float *)malloc(ns * sizeof(float));
    w = (float *)malloc(ns * sizeof(float));
    if (!y || !w || read_bin("projection_n0", y, ns) || read_bin("weight_n0", w, ns)) goto out;
    rc = xtg_upload_sino(ctx, y, w, d);
  } else {
    const int mxy = (int)P->delta_xy, mz = (int)P->delta_z;
    const size_t nb = (size_t)N_r * mxy * N_t * mz;
    y = (float *)malloc(nb * sizeof(float));        /* bright */
    w = (float *)malloc(nb * N_p * sizeof(float));  /* counts */
    if (!y || !w || read_bin("bright_n0", y, nb) || read_bin("weight_n0", w, nb * N_p)) goto out;
    const char *bh = getenv("XT_BH_QUAD_COEF");
    rc = xtg_upload_counts(ctx, y, w, bh ? atof(bh) : 0.0, d);
  }
  if (rc) logf_("ERROR: %s\n", xtg_last_error());
out:
  if (rc && !y) logf_("ERROR: out of host memory or unreadable input\n");
  free(d);
  free(t);
  free(y);
  free(w);
  return rc;
}

/* initObject (XT_ICD_update.c:443-536) with initICD 1 / 2 / 3: the object of
 * this or the coarser stage, upsampled on the GPU with the reference's
 * bilinear schemes (upsample_object_bilinear_2D / _3D, XT_ICD_update.c:354-436),
 * and with --initMagUpMap the magnitude-update map (upsample_bilinear_2D of
 * each (frame, z-block) plane, XT_ICD_update.c:318-352). */
static int load_object(xtg_ctx *ctx, const xt_params *P, const int32_t *dims) {
  const int N_x = dims[0], N_y = dims[1], N_z = dims[2], N_time = dims[3], nzb = dims[7];
  const size_t vol = (size_t)N_z * N_y * N_x, nmag = (size_t)N_time * nzb * N_y * N_x;
  const int sxy = P->initICD >= 2 ? 2 : 1, sz = P->initICD == 3 ? 2 : 1;
  const size_t cvol = (size_t)(N_z / sz) * (N_y / sxy) * (N_x / sxy);
  float *x = (float *)calloc(vol * N_time, sizeof(float));
  float *t = sxy > 1 ? (float *)calloc(cvol * N_time, sizeof(float)) : NULL;
  float *m = NULL;
  int rc = -1;
  char name[256];
  if (!x || (sxy > 1 && !t)) goto out;
  for (int i = 0; i < N_time; i++) {
    snprintf(name, sizeof(name), "object_n0_time_%d", i);
    if (read_bin(name, sxy > 1 ? t + (size_t)i * cvol : x + (size_t)i * vol, sxy > 1 ? cvol : vol)) goto out;
  }
  if (sxy > 1 && xtg_upsample(ctx, t, x, N_time, N_z / sz, N_y / 2, N_x / 2, sz > 1)) goto gpu_err;
  if (xtg_upload_object(ctx, x)) goto gpu_err;
  if (P->initMagUpMap) {
    m = (float *)calloc(nmag, sizeof(float));
    if (!m) goto out;
    if (P->initICD == 1) {
      if (read_bin("mag_update_map_n0", m, nmag)) goto out;
    } else {
      const size_t half = (size_t)N_time * nzb * (N_y / 2) * (N_x / 2);
      free(t);
      t = (float *)calloc(half, sizeof(float));
      if (!t || read_bin("mag_update_map_n0", t, half)) goto out;
      if (xtg_upsample(ctx, t, m, N_time * nzb, 1, N_y / 2, N_x / 2, 0)) goto gpu_err;
    }
    if (xtg_set_magmap(ctx, m)) goto gpu_err;
  }
  rc = 0;
  goto out;
gpu_err:
  logf_("ERROR: %s\n", xtg_last_error());
out:
  free(x);
  free(t);
  free(m);
  return rc;
}

int main(int argc, char **argv) {
  xt_params P;
  xt_engine_opts O;
  if (xt_cli_parse(argc, argv, &P, &O)) return 0;
  g_dbl = P.real_is_double;
  const double t_start = now_s();
  if (!O.quiet) printf("Running.....\n");
  char dbg[256];
  if (P.readSino4mHDF)
    snprintf(dbg, sizeof(dbg), "DEBUG_HDF_Read_n0.log");
  else
    snprintf(dbg, sizeof(dbg), "DEBUG_n0_delta_xy_%d_delta_z_%d.log", (int)P.delta_xy, (int)P.delta_z);
  g_log = fopen(dbg, "w");
  if (!O.quiet) printf("Refer to %s for more information\n", dbg);
  logf_("argsParser: p = %.2f, sigma_s = %f, sigma_t = %f, c_s = %f, c_t = %f, mult_xy = %f, mult_z = %f, "
        "Length_R = %.2f, Length_T = %.2f, stop threshold = %.2f, number of iterations = %d, center of rotation = "
        "%.2f, alpha = %.2f, sinobin = %d, initICD = %d, Rtime0 = %f, Rtime_delta = %f, Rtime_num = %d, N_p = %d, "
        "N_r = %d, N_t = %d, radius_obj = %f, updateProjOffset = %d, no_NHICD = %d, zingerT = %f, zingerDel = %f, "
        "do_VarEst = %d, Est_of_Var = %f, positivity = %d, real_is_double = %d\n",
        P.p, P.sigma_s, P.sigma_t, P.c_s, P.c_t, P.delta_xy, P.delta_z, P.length_r, P.length_t, P.voxel_thresh,
        P.iter, P.rotation_center, P.alpha, P.sinobin, P.initICD, P.Rtime0, P.Rtime_delta, P.Rtime_num,
        P.num_projections, P.N_r, P.N_t, P.radius_obj, P.updateProjOffset, P.no_NHICD, P.zingerT, P.zingerDel,
        P.do_VarEst, P.Est_of_Var, P.positivity, P.real_is_double);
  if (P.readSino4mHDF) {
    logf_("ERROR: reading the sinogram from HDF5 is not part of this engine (no libhdf5); write "
          "projection_n0.bin and weight_n0.bin (or bright_n0.bin and weight_n0.bin) instead\n");
    fprintf(stderr, "ERROR: --readSino4mHDF is not supported; provide .bin inputs\n");
    return 1;
  }
  if (P.sinobin != 1 && P.sinobin != 3) {
    logf_("ERROR: computeWriteSinogram: Cannot recognize sinobin value\n");
    printf("ERROR: computeWriteSinogram: Cannot recognize sinobin value\n");
    return 1;
  }
  if (P.only_Edge_Updates) logf_("WARNING: --only_Edge_Updates is not supported; all voxels in radius_obj are updated\n");
  if (P.initICD > 3 || P.initICD < 0) {
    logf_("ERROR: initObject: initICD value not recognized\n");
    return 1;
  }
  /* variance estimate of the previous stage (XT_Init.c:286-290) */
  if (P.initICD != 0) {
    float v = 0;
    if (read_bin("variance_estimate_n0", &v, 1)) return 1;
    P.Est_of_Var = v;
  }
  double *times = NULL, *angles = NULL;
  char err[512];
  const int32_t nv = xt_read_view_file("view_info.txt", &times, &angles, err, sizeof(err));
  if (nv < 0) {
    logf_("%s\n", err);
    fprintf(stderr, "%s\n", err);
    if (g_log) fclose(g_log);
    return 1;
  }
  /* initSparseAnglesfrmFile's count check, XT_Init.c:158-161 */
  if (nv != P.num_projections) {
    logf_("ERROR: Number of projections read is %d and expected is %d\n", nv, P.num_projections);
    fprintf(stderr, "ERROR: view_info.txt holds %d views, --num_projections is %d\n", nv, P.num_projections);
    free(times);
    free(angles);
    if (g_log) fclose(g_log);
    return 1;
  }
  xtg_ctx *ctx = NULL;
  int rc = xtg_create(&P, times, angles, nv, &ctx);
  free(times);
  free(angles);
  if (rc) {
    logf_("ERROR: %s\n", xtg_last_error());
    fprintf(stderr, "ERROR: %s\n", xtg_last_error());
    return 1;
  }
  rc = xtg_set_options(ctx, O.a_mode, O.sequential ? XTG_ORDER_SEQUENTIAL : XTG_ORDER_PARALLEL,
                       O.columns, O.seed);
  if (rc) {
    logf_("ERROR: %s\n", xtg_last_error());
    goto fail;
  }
  int32_t dims[11];
  xtg_dims(ctx, dims);
  const int N_x = dims[0], N_y = dims[1], N_z = dims[2], N_time = dims[3], nzb = dims[7];
  xt_geom G;
  xtg_geometry(ctx, &G);
  logf_("initStructures: Number of z blocks is %d\n", nzb);

  /* sinogram (genSinogram_fromBin / genSinogram_subsampleCounts) and offset */
  if (load_sinogram(ctx, &P, dims)) goto fail;
  if (P.dont_reconstruct) {
    logf_("XT_Engine: --dont_reconstruct given, no reconstruction\n");
    xtg_destroy(ctx);
    if (g_log) fclose(g_log);
    return 0;
  }
  const size_t nmag = (size_t)N_time * nzb * N_y * N_x;
  if (P.initICD >= 1 && load_object(ctx, &P, dims)) goto fail;

  /* e = y - A x - d, then the cost before ICD (XT_ICD_update.c:998-1007);
   * with initICD 0 the zero start can be replaced by the learned, the
   * multi-resolution or the FBP start */
  if (P.initICD == 0 && O.learned[0]) {
    xtc_net *net = NULL;
    int32_t used = 0;
    double cn = 0, cb = 0;
    rc = xtc_net_create(1, &net);
    if (!rc) rc = xtc_net_load(net, O.learned);
    if (!rc) rc = xtg_init_object_learned(ctx, net, O.multires_iters > 0 ? O.multires_iters : 30, &used, &cn, &cb);
    if (!rc)
      logf_("XT_Engine: learned start %s (network start cost %f, multi-resolution start cost %f)\n",
            used ? "used" : "not lower in cost, multi-resolution start kept", cn, cb);
    xtc_net_destroy(net);
  } else if (P.initICD == 0 && O.multires_iters > 0) {
    rc = xtg_init_object_multires(ctx, O.multires_iters, N_z % 2 == 0 && N_z >= 16);
  } else if (P.initICD == 0 && O.fbp_start) {
    rc = xtg_init_object_fbp(ctx);
  } else {
    rc = xtg_init_error_sino(ctx);
  }
  if (rc) {
    logf_("ERROR: %s\n", xtg_last_error());
    goto fail;
  }
  double cost = 0, fwd = 0, prior = 0;
  if ((rc = xtg_map_cost_fp64(ctx, &cost, &fwd, &prior))) {
    logf_("ERROR: %s\n", xtg_last_error());
    goto fail;
  }
  logf_("costCompute: forward cost=%f\ncostCompute: prior cost =%f\n", fwd, prior);
  logf_("-------------ICD_BackProject: ICD Iter=Before ICD, cost=%f------------\n", cost);
  write_scalar("cost_n0", cost, "wb");
  double cost_last = cost;
  const double t_icd = now_s();
  long long vox_updates = 0;
  int Iter;
  for (Iter = 1; Iter <= P.iter; Iter++) {
    xtg_stats st;
    if ((rc = xtg_icd_iteration(ctx, Iter, &st))) {
      logf_("ERROR: %s\n", xtg_last_error());
      fprintf(stderr, "ERROR: %s\n", xtg_last_error());
      goto fail;
    }
    vox_updates += st.voxel_updates;
    logf_("updateVoxelsTimeSlices: Average voxel update over all voxels is %f, total voxels is %f\n",
          st.total_pix > 0 ? st.mag_sum / st.total_pix : 0.0, st.total_pix);
    logf_("updateVoxelsTimeSlices: Zero count is %lld\n", (long long)st.zero_skipped);
    logf_("updateVoxelsTimeSlices: percentage change in average magnitude is %f\n", st.avg_update_pct);
    if (P.WritePerIter && write_outputs(ctx, dims)) goto fail;
    if (O.resync_every > 0 && Iter % O.resync_every == 0)
      rc = xtg_resync_fp64(ctx, &cost, &fwd, &prior);
    else
      rc = xtg_map_cost_running(ctx, &cost, &fwd, &prior);
    if (rc) {
      logf_("ERROR: %s\n", xtg_last_error());
      goto fail;
    }
    double var = 0;
    xtg_get_variance(ctx, &var);
    logf_("costCompute: forward cost=%f\ncostCompute: prior cost =%f\n", fwd, prior);
    logf_("costCompute: variance parameter estimate =%f\n", var);
    logf_("-------------ICD_BackProject: ICD Iter=%d, cost=%f, time since start of ICD = %fmins------------\n", Iter,
          cost, (now_s() - t_icd) / 60.0);
    logf_("XT_Engine: iteration %d gpu_ms %.3f voxel_updates %lld columns %lld\n", Iter, st.ms,
          (long long)st.voxel_updates, (long long)st.columns);
    write_scalar("cost_n0", cost, "ab");
    if (cost > cost_last) {
      if (!O.quiet) printf("ERROR: ICD_BackProject: Cost value increased\n");
      logf_("ERROR: ICD_BackProject: Cost value increased\n");
    }
    cost_last = cost;
    if (st.converged && Iter > 1) {
      logf_("ICD_BackProject: Convergence criteria is met\n");
      break;
    }
  }
  double var = 0;
  xtg_get_variance(ctx, &var);
  logf_("ICD_BackProject: The estimated variance is %f\n", var);
  write_scalar("variance_estimate_n0", var, "wb");
  float *m = (float *)malloc(sizeof(float) * nmag);
  if (!m || xtg_get_magmap(ctx, m) || write_bin("mag_update_map_n0", m, nmag, "wb")) {
    logf_("ERROR: writing mag_update_map_n0.bin failed\n");
    free(m);
    goto fail;
  }
  free(m);
  if (write_outputs(ctx, dims)) goto fail;
  const double t_end = now_s();
  logf_("XT_Engine: done, %d iterations, %lld voxel updates, ICD %.3f s, total %.3f s\n",
        Iter > P.iter ? P.iter : Iter, vox_updates, t_end - t_icd, t_end - t_start);
  if (!O.quiet) printf("Program will exit now\n");
  xtg_destroy(ctx);
  if (g_log) fclose(g_log);
  (void)G;
  return 0;
fail:
  xtg_destroy(ctx);
  if (g_log) fclose(g_log);
  return 1;
}
