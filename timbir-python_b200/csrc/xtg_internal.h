// xtg_internal.h -- declarations shared by the .cu files of libxtgpu.
#pragma once
#include "xtg_kernels.cuh"

namespace xtg {

struct IcdArgs {
  float *e;
  const float *w;
  float *x;
  float *magmap;
  const float *hr, *cosv, *sinv;
  const int *view_idx, *view_start, *view_num;
  const int4 *items;
  const int *n_items_dev;  // device item count (NHICD lists), or null
  int n_items;             // host item count when n_items_dev is null
  int item_lo;             // first item index of this launch
  int *counter;
  int use_perm;
  unsigned long long perm_key;
  const uint4 *a16;        // FP16 A records [frame][col_rank][vmax] or null
  const float *a16_scale;  // [frame][col_rank]
  const int *col_rank;     // [N_y*N_x] -> rank in the masked list, -1 outside
  int a16_vmax, n_masked;
  int iter;
  float T2, Tdelta;
  double *st_absx;             // [64] slots
  unsigned long long *st_cnt;  // [0] voxel updates, [1] zero skipped, [2] items
  int *err;
};

size_t icd_smem_bytes(int vmax, int zmax, int zovl, int as);
cudaError_t launch_icd(const DevGeo &G, const IcdArgs &A, int vec, int amode, int seq, int as, int vmax, int zmax,
                       int grid, cudaStream_t st);
int icd_occupancy(int vec, int amode, int seq, int as, int vmax, int zmax, int zovl);

}  // namespace xtg
