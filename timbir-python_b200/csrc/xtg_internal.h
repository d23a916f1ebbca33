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
  // z-slab split: base item i is processed as nsub pieces of at most zslab
  // slices; the launch visits piece-major (all items' piece 0, then piece 1,
  // ...), so the detector rows in flight stay within one slab of e and w
  int zslab, nsub;
  // A column table (a_mode FP16 / FP32 table): entries of (frame, masked
  // column rank) at [tstart[i], tstart[i+1]), i = frame * n_masked + rank
  const long long *tstart;
  const int *toff;          // (p * N_r + bin) * N_t of each entry
  const float *tval32;      // A * delta_t (FP32 table)
  const __half *tval16;     // A * delta_t / scale (FP16 table)
  const float *tscale;      // per (frame, column) scale of the FP16 table
  const int *col_rank;      // [N_y*N_x] -> rank in the masked list, -1 outside
  int n_masked;
  int w_keep;  // e and w fit in L2 together: w loads keep their lines (evict_last)
  int iter;
  float T2, Tdelta;
  // z slab of a larger volume: the neighbouring slabs' boundary slices,
  // [N_time][N_y][N_x] (null where this slab ends the volume)
  const float *halo_lo, *halo_hi;
  double *st_absx;             // [64] slots
  unsigned long long *st_cnt;  // [0] voxel updates, [1] zero skipped, [2] items
  int *err;
};

#define FP_WARPS 4  // warps per projector CTA, 32 detector bins each

struct FpArgs {
  const float *x, *y, *d, *w, *hr, *cosv, *sinv;
  const int *fov;
  float *out;          // ax (mode 0) or e (modes 1, 2)
  double *cost_slots;  // modes 2, 3: 64 slots
  float T;
  float delta;
  double win_margin;
};

// bin-major A table: row (view p, bin r) = entries [ptr[p N_r + r], ptr[p N_r + r + 1])
struct CsrBuildArgs {
  const float *hr, *cosv, *sinv;
  double win_margin;
  int *count;           // build pass 0: entries per row
  const long long *ptr; // build pass 1: row starts
  int2 *ent;            // {(j * N_x + k) * N_z, bits of its A (without delta_t)} per entry
};
struct CsrView {
  const long long *ptr;
  const int2 *ent;
};

struct TableArgs {
  const float *hr, *cosv, *sinv;
  const int *view_idx, *view_start, *view_num, *mcols;
  int n_masked;
  const long long *start;
  int *off;
  float *val32;
  __half *val16;
  float *scale;
};

cudaError_t launch_fp(const DevGeo &G, const FpArgs &F, int mode, int ns, cudaStream_t st);
cudaError_t launch_csr_build(const DevGeo &G, const CsrBuildArgs &B, int fill, int ns, cudaStream_t st);
cudaError_t launch_fp_csr(const DevGeo &G, const FpArgs &F, const CsrView &T, int mode, cudaStream_t st);
cudaError_t launch_table_count(const DevGeo &G, const TableArgs &T, int ns, long long *count, cudaStream_t st);
cudaError_t launch_table_fill(const DevGeo &G, const TableArgs &T, int ns, cudaStream_t st);

size_t icd_smem_bytes(int vmax, int zmax, int zovl, int as, int amode, int vec, int nt);
cudaError_t launch_fbp(const DevGeo &G, const float *y, const float *d, float *q, const float *cosv,
                       const float *sinv, const int *view_idx, const int *view_start, const int *view_num,
                       const int *col_rank, float *x, cudaStream_t st);
cudaError_t launch_magmap_zero(const DevGeo &G, const IcdArgs &A, int grid, cudaStream_t st);
cudaError_t launch_icd(const DevGeo &G, const IcdArgs &A, int vec, int amode, int seq, int as, int vmax, int zmax,
                       int grid, cudaStream_t st);
int icd_occupancy(int vec, int amode, int seq, int as, int vmax, int zmax, int zovl);

}  // namespace xtg
