/*
 * xt_cli.c -- XT_Engine command-line parser (see xt_cli.h).
 */
#define _GNU_SOURCE
#include "xt_cli.h"
#include "xtg.h"

#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { OPT_POS = 300, OPT_DOUBLE, OPT_AFP16, OPT_SEQ, OPT_COLS, OPT_SEED, OPT_RESYNC, OPT_QUIET, OPT_HELP, OPT_AMODE, OPT_FBP, OPT_MULTIRES, OPT_LEARNED };

int xt_cli_parse(int argc, char **argv, xt_params *p, xt_engine_opts *o) {
  /* option table of XT_Init.c:457-506: names, letters and argument kinds */
  static struct option opts[] = {
      {"p", required_argument, 0, 'a'},
      {"sigma_s", required_argument, 0, 'b'},
      {"c_s", required_argument, 0, 'c'},
      {"sigma_t", required_argument, 0, 'd'},
      {"c_t", required_argument, 0, 'e'},
      {"delta_xy", required_argument, 0, 'f'},
      {"delta_z", required_argument, 0, 'z'},
      {"length_r", required_argument, 0, 'g'},
      {"num_threads", required_argument, 0, 'h'},
      {"length_t", required_argument, 0, '3'},
      {"voxel_thresh", required_argument, 0, 'j'},
      {"iter", required_argument, 0, 'k'},
      {"rotation_center", required_argument, 0, 'l'},
      {"alpha", required_argument, 0, 'm'},
      {"time_reg", no_argument, 0, 'n'},
      {"sinobin", required_argument, 0, 'o'},
      {"initICD", required_argument, 0, 'p'},
      {"writeTiff", required_argument, 0, 'q'},
      {"NoNoise", no_argument, 0, 'r'},
      {"Rtime0", required_argument, 0, 's'},
      {"Rtime_delta", required_argument, 0, 't'},
      {"Rtime_num", required_argument, 0, 'u'},
      {"num_projections", required_argument, 0, 'v'},
      {"N_r", required_argument, 0, 'w'},
      {"dont_reconstruct", no_argument, 0, 'x'},
      {"cost_thresh", required_argument, 0, 'y'},
      {"radius_obj", required_argument, 0, 'i'},
      {"detector_slice_begin", required_argument, 0, '1'},
      {"detector_slice_num", required_argument, 0, '2'},
      {"phantom_N_xy", required_argument, 0, '4'},
      {"phantom_N_z", required_argument, 0, '5'},
      {"N_t", required_argument, 0, '6'},
      {"updateProjOffset", required_argument, 0, '7'},
      {"EnforceZeroMeanOffset", no_argument, 0, '#'},
      {"no_NHICD", no_argument, 0, '8'},
      {"WritePerIter", no_argument, 0, '+'},
      {"only_Edge_Updates", no_argument, 0, '-'},
      {"zingerT", required_argument, 0, '*'},
      {"zingerDel", required_argument, 0, '^'},
      {"initMagUpMap", no_argument, 0, '&'},
      {"readSino4mHDF", no_argument, 0, '>'},
      {"do_VarEst", no_argument, 0, '%'},
      {"Est_of_Var", required_argument, 0, '('},
      {"RMSE_converged", no_argument, 0, ';'},
      {"x_start", required_argument, 0, '['},
      {"x_width", required_argument, 0, ']'},
      /* this engine's own options */
      {"positivity", required_argument, 0, OPT_POS},
      {"real_is_double", no_argument, 0, OPT_DOUBLE},
      {"gpu_afp16", no_argument, 0, OPT_AFP16},
      {"gpu_amode", required_argument, 0, OPT_AMODE},
      {"gpu_fbp_start", no_argument, 0, OPT_FBP},
      {"gpu_multires_start", required_argument, 0, OPT_MULTIRES},
      {"gpu_learned_start", required_argument, 0, OPT_LEARNED},
      {"gpu_sequential", no_argument, 0, OPT_SEQ},
      {"gpu_columns", required_argument, 0, OPT_COLS},
      {"gpu_seed", required_argument, 0, OPT_SEED},
      {"gpu_resync", required_argument, 0, OPT_RESYNC},
      {"quiet", no_argument, 0, OPT_QUIET},
      {"help", no_argument, 0, OPT_HELP},
      {0, 0, 0, 0}};
  xt_params_default(p);
  memset(o, 0, sizeof(*o));
  o->seed = 761521;
  o->a_mode = XTG_A_AUTO;
  o->resync_every = 10;
  optind = 0;
  for (;;) {
    int idx = 0;
    const int c = getopt_long(argc, argv, "a:b:c:d:e:f:z:g:h:3:j:k:l:m:no:p:q:rs:t:u:v:w:xy:i:1:2:4:5:6:7:#8+-*:^:&>%(:;[:]:",
                              opts, &idx);
    if (c == -1) break;
    switch (c) {
      case 'a': p->p = atof(optarg); break;
      case 'b': p->sigma_s = atof(optarg); break;
      case 'c': p->c_s = atof(optarg); break;
      case 'd': p->sigma_t = atof(optarg); break;
      case 'e': p->c_t = atof(optarg); break;
      case 'f': p->delta_xy = atof(optarg); break;
      case 'z': p->delta_z = atof(optarg); break;
      case 'g': p->length_r = atof(optarg); break;
      case 'h': p->num_threads = atoi(optarg); break;
      case '3': p->length_t = atof(optarg); break;
      case 'j': p->voxel_thresh = atof(optarg); break;
      case 'k': p->iter = atoi(optarg); break;
      case 'l': p->rotation_center = atof(optarg); break;
      case 'm': p->alpha = atof(optarg); break;
      case 'n': p->time_reg = 1; break;
      case 'o': p->sinobin = atoi(optarg); break;
      case 'p': p->initICD = atoi(optarg); break;
      case 'q': p->writeTiff = atoi(optarg); break;
      case 'r': p->NoNoise = 1; break;
      case 's': p->Rtime0 = atof(optarg); break;
      case 't': p->Rtime_delta = atof(optarg); break;
      case 'u': p->Rtime_num = atoi(optarg); break;
      case 'v': p->num_projections = atoi(optarg); break;
      case 'w': p->N_r = atoi(optarg); break;
      case 'x': p->dont_reconstruct = 1; break;
      case 'y': p->cost_thresh = atof(optarg); break;
      case 'i': p->radius_obj = atof(optarg); break;
      case '1': p->detector_slice_begin = atoi(optarg); break;
      case '2': p->detector_slice_num = atoi(optarg); break;
      case '4': p->phantom_N_xy = atoi(optarg); break;
      case '5': p->phantom_N_z = atoi(optarg); break;
      case '6': p->N_t = atoi(optarg); break;
      case '7': p->updateProjOffset = atoi(optarg); break;
      case '#': p->EnforceZeroMeanOffset = 1; break;
      case '8': p->no_NHICD = 1; break;
      case '+': p->WritePerIter = 1; break;
      case '-': p->only_Edge_Updates = 1; break;
      case '*': p->zingerT = atof(optarg); break;
      case '^': p->zingerDel = atof(optarg); break;
      case '&': p->initMagUpMap = 1; break;
      case '>': p->readSino4mHDF = 1; break;
      case '%': p->do_VarEst = 1; break;
      case '(': p->Est_of_Var = atof(optarg); break;
      case ';': p->RMSE_converged = 1; break;
      case '[': p->x_start = atoi(optarg); break;
      case ']': p->x_width = atoi(optarg); break;
      case OPT_POS: p->positivity = atoi(optarg) != 0; break;
      case OPT_DOUBLE: p->real_is_double = 1; break;
      case OPT_AFP16: o->a_mode = XTG_A_FP16; break;
      case OPT_AMODE:
        if (!strcmp(optarg, "fp32")) o->a_mode = XTG_A_FP32;
        else if (!strcmp(optarg, "table32")) o->a_mode = XTG_A_TABLE32;
        else if (!strcmp(optarg, "fp16")) o->a_mode = XTG_A_FP16;
        else if (!strcmp(optarg, "auto")) o->a_mode = XTG_A_AUTO;
        else printf("ERROR: XT_Engine: --gpu_amode takes fp32, table32, fp16 or auto; keeping the default\n");
        break;
      case OPT_SEQ: o->sequential = 1; break;
      case OPT_FBP: o->fbp_start = 1; break;
      case OPT_MULTIRES: o->multires_iters = atoi(optarg); break;
      case OPT_LEARNED: snprintf(o->learned, sizeof o->learned, "%s", optarg); break;
      case OPT_COLS: o->columns = atoi(optarg); break;
      case OPT_SEED: o->seed = strtoull(optarg, NULL, 10); break;
      case OPT_RESYNC: o->resync_every = atoi(optarg); break;
      case OPT_QUIET: o->quiet = 1; break;
      case OPT_HELP:
        printf("XT_Engine: TIMBIR/MBIR reconstruction on one B200; options as the reference XT_Engine,\n"
               "plus --positivity 0|1 --real_is_double --gpu_amode fp32|table32|fp16|auto --gpu_afp16\n"
               "--gpu_fbp_start --gpu_multires_start N --gpu_learned_start WEIGHTS --gpu_sequential --gpu_columns N\n"
               "--gpu_seed S --gpu_resync K --quiet\n");
        return 1;
      default:
        /* the reference reports and carries on (XT_Init.c:590) */
        printf("ERROR: argsParser: Cannot recognize argument %s\n", optarg ? optarg : "");
        o->n_unknown++;
        break;
    }
  }
  return 0;
}
