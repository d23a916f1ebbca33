// xtg_proj.cu -- forward projection and the A-matrix column table.
//
// Forward projection (initErrorSinogam + forward_project_voxel_AMat1D,
// Source_Code_4D_Fast/XT_ICD_update.c:551-569, XT_ForwardProject.c:8-25) as a
// gather: one warp per (view, 32 detector bins, 64 detector rows), partial
// sums in shared memory owned by that warp.  The warp walks image rows in
// increasing order and, within a row, the columns that can reach its bins in
// increasing order, so every sinogram entry is summed in the reference's
// (row, column) order: the FP32 result is bit-identical to the reference's,
// and FP64 accumulation gives the resync / MAP-cost data term.
//
// A-matrix column table (calcAMatrixColumnforAngle, XT_AMatrix.c:50-110,
// for every masked column and every view of its frame, stored once): CSC
// form, per (frame, column) a run of entries {offset (p*N_r + bin)*N_t,
// A*delta_t} in view order, FP32 or FP16 with one FP32 scale per column.
// The ICD kernel streams these runs instead of recomputing A per visit.
#include <cuda_fp16.h>

#include "xtg_internal.h"

namespace xtg {

// candidate columns of row yv for bin window [lo, hi] of r_col (conservative)
__device__ __forceinline__ bool fp_col_range(const DevGeo &G, float cp, float sp, float yv, double lo, double hi,
                                             int *klo, int *khi) {
  const double ys = (double)yv * (double)sp;
  if (fabs((double)cp) < 1e-12) {
    if (-ys >= lo && -ys <= hi) {
      *klo = 0;
      *khi = G.N_x - 1;
      return true;
    }
    return false;
  }
  double xa = (lo + ys) / (double)cp, xb = (hi + ys) / (double)cp;
  if (xa > xb) {
    const double t = xa;
    xa = xb;
    xb = t;
  }
  const double ka = (xa - (double)G.x0) / (double)G.delta_xy - 0.5;
  const double kb = (xb - (double)G.x0) / (double)G.delta_xy - 0.5;
  if (kb < -4.0 || ka > (double)G.N_x + 4.0) return false;
  *klo = max(0, (int)floor(ka) - 2);
  *khi = min(G.N_x - 1, (int)ceil(kb) + 2);
  return *klo <= *khi;
}

// MODE 0: out = A x; 1: out = e = y - A x - d (FP32, the reference's order
// and its projector, which leaves out delta_t, XT_ForwardProject.c:17);
// 2: FP64 sums, out = (float)(y - delta_t A x - d), data cost into cost slots;
// 3: FP64 data cost only.  Modes 2 and 3 use A * delta_t, the matrix the
// voxel update subtracts from e (XT_VoxUpdate.c:27, 67): the error sinogram
// the reference carries from its zero start; with delta_t = 1 all modes agree.
// Warp w of the CTA owns 32 consecutive detector bins of view p and keeps
// their partial sums for 64 detector rows in shared memory (lane owns rows
// lane and lane + 32, so the shared accesses are free of bank conflicts).  For each image row (in increasing order) the warp
// evaluates, one column per lane, the exact A entries of the columns that can
// reach its bins, then walks those columns in increasing order: one
// coalesced z-line load per column, and each of the column's entries that
// falls on the warp's bins is added with a plain shared-memory read-add-write
// (the warp owns those sums, so no atomics).  Control flow is uniform within
// the warp.
template <int MODE, typename ACC, int NS>
__global__ void __launch_bounds__(FP_WARPS * 32) k_fp_bins(DevGeo G, FpArgs F) {
  extern __shared__ __align__(16) unsigned char fp_sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  ACC *acc = reinterpret_cast<ACC *>(fp_sm) + (size_t)warp * 32 * 64;  // [32 bins][64 rows]
  // the A entries of the warp's 32 candidate columns, [lane][NS]
  float *vsm = reinterpret_cast<float *>(fp_sm + (size_t)FP_WARPS * 32 * 64 * sizeof(ACC)) + (size_t)warp * 32 * NS;
  const int p = blockIdx.x;
  const int rb = (blockIdx.y * FP_WARPS + warp) * 32;
  const int t0 = blockIdx.z * 64, nt = min(64, G.N_t - t0);
  if (rb >= G.N_r) return;  // whole warp; no block-wide barrier follows
#pragma unroll 4
  for (int b = 0; b < 32; b++) {
    acc[b * 64 + lane] = (ACC)0;
    acc[b * 64 + lane + 32] = (ACC)0;
  }
  __syncwarp();
  const int fr = F.fov[p];
  const float cp = F.cosv[p], sp = F.sinv[p];
  const float *H = F.hr + (size_t)p * XT_HR_STRIDE;
  const double lo = (double)G.R0 + (double)rb * G.delta_r - G.delta_xy - F.win_margin;
  const double hi = (double)G.R0 + (double)(rb + 32) * G.delta_r + G.delta_xy + F.win_margin;
  const int ta = lane, tb = lane + 32;  // this lane's rows (relative to t0)
  // slices of those rows (detector row t belongs to slice t / zovl)
  const bool va = ta < nt, vb = tb < nt;
  const int za = (t0 + ta) / G.zovl, zb2 = (t0 + tb) / G.zovl;
  for (int j = 0; j < G.N_y; j++) {
    int klo, khi;
    if (!fp_col_range(G, cp, sp, xt_coord(G.y0, j, G.delta_xy), lo, hi, &klo, &khi)) continue;
    const float *xrow = F.x + ((size_t)fr * G.N_y + j) * G.N_x * G.N_z;
    for (int kb = klo; kb <= khi; kb += 32) {
      const int k = kb + lane;
      float v[NS];
#pragma unroll
      for (int s = 0; s < NS; s++) v[s] = 0.f;
      int first = 0, n = 0;
      if (k <= khi) n = xt_amatrix_regs<NS>(G, H, cp, sp, j, k, v, &first);
      // entries of this lane's column that land on the warp's bins
      const int slo = max(0, rb - first), shi = min(n, rb + 32 - first);
      const unsigned hit = __ballot_sync(0xffffffffu, slo < shi);
      if (!hit) continue;
      // each column's entries go to shared memory, its (first - rb, slo, shi)
      // into one word, so a hit column costs one shuffle and its entries that
      // land on the warp's bins are read by a loop over exactly those
#pragma unroll
      for (int s = 0; s < NS; s++) vsm[lane * NS + s] = v[s];
      // for a hit column first - rb lies in (-NS, 32), so the +64 keeps it positive
      const int pk = (int)(((unsigned)(first - rb + 64) << 16) | ((unsigned)slo << 8) | (unsigned)shi);
      __syncwarp();
      unsigned mk = hit;
      // the z-line of the next hit column is loaded while the current one is added
      float xa = 0.f, xb = 0.f;
      {
        const float *xp = xrow + (size_t)(kb + __ffs(mk) - 1) * G.N_z;
        xa = va ? __ldg(xp + za) : 0.f;
        xb = vb ? __ldg(xp + zb2) : 0.f;
      }
      while (mk) {
        const int l = __ffs(mk) - 1;
        mk &= mk - 1;
        const int q = __shfl_sync(0xffffffffu, pk, l);
        const int sl = (q >> 8) & 0xFF, sh = q & 0xFF;
        const float ca = xa, cb = xb;
        if (mk) {
          const float *xp = xrow + (size_t)(kb + __ffs(mk) - 1) * G.N_z;
          xa = va ? __ldg(xp + za) : 0.f;
          xb = vb ? __ldg(xp + zb2) : 0.f;
        }
        ACC *qa = acc + ((q >> 16) - 64 + sl) * 64;
        const float *vl = vsm + l * NS;
        for (int s = sl; s < sh; s++, qa += 64) {
          const float a = vl[s];
          if (a != 0.f) {
            if (MODE <= 1) {
              qa[ta] = __fadd_rn(qa[ta], __fmul_rn(ca, a));
              qa[tb] = __fadd_rn(qa[tb], __fmul_rn(cb, a));
            } else {
              qa[ta] += (ACC)ca * (ACC)a;
              qa[tb] += (ACC)cb * (ACC)a;
            }
          }
        }
      }
      __syncwarp();  // the staged entries are rewritten by the next round
    }
  }
  __syncwarp();
  double cacc = 0.0;
  for (int b = 0; b < 32; b++) {
    const int r = rb + b;
    if (r >= G.N_r) break;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int t = lane + 32 * h;
      if (t >= nt) continue;
      const ACC sacc = acc[b * 64 + t];
      const size_t o = ((size_t)p * G.N_r + r) * G.N_t + t0 + t;
      const size_t od = (size_t)r * G.N_t + t0 + t;
      if (MODE == 0) {
        F.out[o] = (float)sacc;
      } else if (MODE == 1) {
        F.out[o] = __fsub_rn(__fsub_rn(F.y[o], (float)sacc), F.d[od]);
      } else {
        // A * delta_t: the system matrix of the voxel update (XT_VoxUpdate.c:27, 67)
        const double e64 = (double)F.y[o] - (double)G.delta_t * (double)sacc - (double)F.d[od];
        if (MODE == 2) F.out[o] = (float)e64;
        const double sw = e64 * sqrt((double)F.w[o]);
        if (fabs(sw) < (double)F.T)
          cacc += sw * sw;
        else
          cacc += 2.0 * (double)F.delta * (double)F.T * fabs(sw) + (double)F.T * (double)F.T * (1.0 - 2.0 * (double)F.delta);
      }
    }
  }
  if (MODE >= 2) {
    for (int off = 16; off > 0; off >>= 1) cacc += __shfl_xor_sync(0xffffffffu, cacc, off);
    if (lane == 0) atomicAdd(&F.cost_slots[(blockIdx.x * 5 + blockIdx.y * 3 + blockIdx.z + warp) % 64], cacc);
  }
}

template <int MODE, typename ACC>
static cudaError_t launch_fp_t(const DevGeo &G, const FpArgs &F, int ns, cudaStream_t st) {
  const int nsv = ns <= 3 ? 3 : ns <= 4 ? 4 : 12;
  const size_t smem = (size_t)FP_WARPS * 32 * 64 * sizeof(ACC) + (size_t)FP_WARPS * 32 * nsv * sizeof(float);
  dim3 grid((unsigned)G.N_p, (unsigned)((G.N_r + FP_WARPS * 32 - 1) / (FP_WARPS * 32)), (unsigned)((G.N_t + 63) / 64));
  typedef void (*K)(DevGeo, FpArgs);
  K k = ns <= 3 ? k_fp_bins<MODE, ACC, 3> : ns <= 4 ? k_fp_bins<MODE, ACC, 4> : k_fp_bins<MODE, ACC, 12>;
  cudaError_t e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, FP_WARPS * 32, smem, st>>>(G, F);
  return cudaGetLastError();
}

cudaError_t launch_fp(const DevGeo &G, const FpArgs &F, int mode, int ns, cudaStream_t st) {
  switch (mode) {
    case 0: return launch_fp_t<0, float>(G, F, ns, st);
    case 1: return launch_fp_t<1, float>(G, F, ns, st);
    case 2: return launch_fp_t<2, double>(G, F, ns, st);
    default: return launch_fp_t<3, double>(G, F, ns, st);
  }
}

// ------------------------------------------------------- A column table --
// entries of (frame f, masked column ci): one warp, lanes over views
template <int NS>
__global__ void k_table_count(DevGeo G, TableArgs T, long long *count) {
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= (long long)G.N_time * T.n_masked) return;
  const int f = (int)(gw / T.n_masked), c = T.mcols[gw % T.n_masked];
  const int row = c / G.N_x, col = c % G.N_x, V = T.view_num[f], vs = T.view_start[f];
  int n = 0;
  for (int v = lane; v < V; v += 32) {
    const int p = T.view_idx[vs + v];
    float vals[NS];
    int first;
    n += xt_amatrix_regs<NS>(G, T.hr + (size_t)p * XT_HR_STRIDE, T.cosv[p], T.sinv[p], row, col, vals, &first);
  }
  for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
  if (lane == 0) count[gw] = n;
}

template <int NS>
__global__ void k_table_fill(DevGeo G, TableArgs T) {
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= (long long)G.N_time * T.n_masked) return;
  const int f = (int)(gw / T.n_masked), c = T.mcols[gw % T.n_masked];
  const int row = c / G.N_x, col = c % G.N_x, V = T.view_num[f], vs = T.view_start[f];
  float mx = 0.f;
  if (T.val16) {
    for (int v = lane; v < V; v += 32) {
      const int p = T.view_idx[vs + v];
      float vals[NS];
      int first;
      const int n = xt_amatrix_regs<NS>(G, T.hr + (size_t)p * XT_HR_STRIDE, T.cosv[p], T.sinv[p], row, col, vals, &first);
#pragma unroll
      for (int s = 0; s < NS; s++)
        if (s < n) mx = fmaxf(mx, __fmul_rn(vals[s], G.delta_t));
    }
    for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  }
  const float sc = mx > 0.f ? mx : 1.f;
  if (T.val16 && lane == 0) T.scale[gw] = sc;
  long long pos = T.start[gw];
  for (int v0 = 0; v0 < V; v0 += 32) {
    const int v = v0 + lane;
    float vals[NS];
    int first = 0, n = 0;
    if (v < V) {
      const int p = T.view_idx[vs + v];
      n = xt_amatrix_regs<NS>(G, T.hr + (size_t)p * XT_HR_STRIDE, T.cosv[p], T.sinv[p], row, col, vals, &first);
      first = (int)(((long long)p * G.N_r + first) * G.N_t);  // offset of the first entry's rows
    }
    int incl = n;  // inclusive prefix of n over the warp keeps the view order
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += y;
    }
    const long long my = pos + incl - n;
#pragma unroll
    for (int s = 0; s < NS; s++) {
      if (s < n) {
        T.off[my + s] = first + s * G.N_t;
        const float a = __fmul_rn(vals[s], G.delta_t);
        if (T.val16)
          T.val16[my + s] = __float2half_rn(a / sc);
        else
          T.val32[my + s] = a;
      }
    }
    pos += __shfl_sync(0xffffffffu, incl, 31);
  }
}

cudaError_t launch_table_count(const DevGeo &G, const TableArgs &T, int ns, long long *count, cudaStream_t st) {
  const long long warps = (long long)G.N_time * T.n_masked;
  const unsigned grid = (unsigned)((warps + 7) / 8);
  if (ns <= 3)
    k_table_count<3><<<grid, 256, 0, st>>>(G, T, count);
  else if (ns <= 4)
    k_table_count<4><<<grid, 256, 0, st>>>(G, T, count);
  else
    k_table_count<12><<<grid, 256, 0, st>>>(G, T, count);
  return cudaGetLastError();
}

cudaError_t launch_table_fill(const DevGeo &G, const TableArgs &T, int ns, cudaStream_t st) {
  const long long warps = (long long)G.N_time * T.n_masked;
  const unsigned grid = (unsigned)((warps + 7) / 8);
  if (ns <= 3)
    k_table_fill<3><<<grid, 256, 0, st>>>(G, T);
  else if (ns <= 4)
    k_table_fill<4><<<grid, 256, 0, st>>>(G, T);
  else
    k_table_fill<12><<<grid, 256, 0, st>>>(G, T);
  return cudaGetLastError();
}

}  // namespace xtg
