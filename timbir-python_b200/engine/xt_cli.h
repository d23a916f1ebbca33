/*
 * xt_cli.h -- the XT_Engine command line.
 *
 * Same long options, short letters and defaults as the reference's
 * argsParser (Source_Code_4D_Fast/XT_Init.c:452-629), so the launcher's
 * command string (4D_Recon_Launcher_for_Real_Data/XT_MBIR_Reconstruction.py:124-157)
 * runs unchanged.  A few long-only options (values >= 300) select what the
 * reference fixes at compile time or what only the GPU engine has.
 */
#ifndef XT_CLI_H
#define XT_CLI_H
#include <stdint.h>

#include "xt_geom.h"

typedef struct {
  int32_t fbp_start;    /* --gpu_fbp_start: with initICD 0, start from the FBP image instead of zero */
  int32_t multires_iters; /* --gpu_multires_start N: with initICD 0, the multi-resolution start with N coarse iterations */
  char learned[512];    /* --gpu_learned_start PATH: with initICD 0, the learned start with these weights */
  int32_t a_mode;       /* --gpu_amode fp32|table32|fp16|auto (XTG_A_*); --gpu_afp16 = fp16 */
  int32_t sequential;   /* --gpu_sequential: reference visiting order, one column at a time */
  int32_t columns;      /* --gpu_columns N: columns in flight (0 = device default) */
  uint64_t seed;        /* --gpu_seed S: seed of the GPU visiting order */
  int32_t resync_every; /* --gpu_resync K: FP64 resync of e every K iterations (default 10);
                           the other iterations take the cost of the running e, in FP64 sums */
  int32_t quiet;        /* --quiet: no stdout chatter */
  int32_t n_unknown;    /* unrecognised options seen (reported, not fatal, like the reference) */
} xt_engine_opts;

/* Parses argv into *p and *o; returns 0, or 1 after printing usage for --help. */
int xt_cli_parse(int argc, char **argv, xt_params *p, xt_engine_opts *o);

#endif
