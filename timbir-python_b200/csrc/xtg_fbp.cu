// xtg_fbp.cu -- filtered backprojection start for ICD.
//
// The reference starts ICD from a zero object (initObject, XT_ICD_update.c:
// 454-458) or from a coarser stage; its launchers compute FBP images with
// scikit-image outside the engine (4D_Recon_Launcher_for_Real_Data/
// XT_FBP_Reconstruction.py).  This is the parallel-beam FBP of Kak & Slaney
// (Principles of Computerized Tomographic Imaging, ch. 3, eqs. 61-63) on the
// engine's own geometry, used as a warm start:
//   q_p(r_k, t) = dr * sum_n h(k - n) (y[p][n][t] - d[n][t]),
//     h(0) = 1 / (4 dr^2), h(m odd) = -1 / (m^2 pi^2 dr^2), h(m even) = 0;
//   x(j, k, z) = (pi / V_f) sum_{views p of the frame} q_p(x cos th - y sin th, t)
// with linear interpolation between bin centres R0 + (i + 0.5) dr and the
// zovl detector rows of slice z averaged.  Columns outside the reconstruction
// disk get 0; with positivity the image is clamped at 0.
#include "xtg_internal.h"

namespace xtg {

#define FBP_TT 32  // detector rows per ramp-filter CTA

// one CTA per (view, 32 detector rows): the view's rows in shared memory,
// warps over bins, lanes over rows
__global__ void __launch_bounds__(256) k_ramp(DevGeo G, const float *__restrict__ y, const float *__restrict__ d,
                                              float *__restrict__ q) {
  extern __shared__ float fbp_sm[];
  float *s = fbp_sm;                            // [N_r][FBP_TT + 1]
  float *h = fbp_sm + (size_t)G.N_r * (FBP_TT + 1);  // h[m] for odd m < N_r, index m / 2
  const int p = blockIdx.x, t0 = blockIdx.y * FBP_TT, nt = min(FBP_TT, G.N_t - t0);
  const double dr = (double)G.delta_r;
  for (int i = threadIdx.x; i < G.N_r * FBP_TT; i += blockDim.x) {
    const int r = i / FBP_TT, tt = i - r * FBP_TT;
    float v = 0.f;
    if (tt < nt) {
      const size_t o = ((size_t)p * G.N_r + r) * G.N_t + t0 + tt;
      v = y[o] - (d ? d[(size_t)r * G.N_t + t0 + tt] : 0.f);
    }
    s[r * (FBP_TT + 1) + tt] = v;
  }
  for (int m = 2 * threadIdx.x + 1; m < G.N_r; m += 2 * blockDim.x)
    h[m / 2] = (float)(-1.0 / ((double)m * m * M_PI * M_PI * dr * dr));
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float h0 = (float)(1.0 / (4.0 * dr * dr));
  for (int r = warp; r < G.N_r; r += nw) {
    float acc = h0 * s[r * (FBP_TT + 1) + lane];
    for (int m = 1; m < G.N_r; m += 2) {
      const float hv = h[m / 2];
      float a = 0.f;
      if (r - m >= 0) a += s[(r - m) * (FBP_TT + 1) + lane];
      if (r + m < G.N_r) a += s[(r + m) * (FBP_TT + 1) + lane];
      acc = fmaf(hv, a, acc);
    }
    if (lane < nt) q[((size_t)p * G.N_r + r) * G.N_t + t0 + lane] = (float)dr * acc;
  }
}

// one warp per (frame, row, column); lanes over detector rows, 128 at a time
__global__ void __launch_bounds__(256) k_backproject(DevGeo G, const float *__restrict__ q,
                                                     const float *__restrict__ cosv, const float *__restrict__ sinv,
                                                     const int *__restrict__ view_idx, const int *__restrict__ view_start,
                                                     const int *__restrict__ view_num, const int *__restrict__ col_rank,
                                                     float *__restrict__ x) {
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long long ncol = (long long)G.N_time * G.N_y * G.N_x;
  if (gw >= ncol) return;
  const int fr = (int)(gw / ((long long)G.N_y * G.N_x));
  const int rem = (int)(gw - (long long)fr * G.N_y * G.N_x);
  const int j = rem / G.N_x, k = rem - j * G.N_x;
  float *xz = x + (size_t)gw * G.N_z;  // [N_time][N_y][N_x][N_z]
  if (col_rank[(size_t)j * G.N_x + k] < 0) {
    for (int z = lane; z < G.N_z; z += 32) xz[z] = 0.f;
    return;
  }
  const float xc = xt_coord(G.x0, k, G.delta_xy), yc = xt_coord(G.y0, j, G.delta_xy);
  const int V = view_num[fr], vs = view_start[fr];
  const float scale = (float)(M_PI / (double)V) / (float)G.zovl;
  // tiles of TR detector rows, TR a multiple of zovl so no slice straddles two
  const int TR = (128 / G.zovl) * G.zovl;
  __shared__ float rows[8][128];
  float *rw = rows[threadIdx.x >> 5];
  for (int tb = 0; tb < G.N_t; tb += TR) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int v = 0; v < V; v++) {
      const int p = view_idx[vs + v];
      const float r = xc * cosv[p] - yc * sinv[p];
      const float u = (r - G.R0) / G.delta_r - 0.5f;
      const float fl = floorf(u);
      const int i = (int)fl;
      const float f = u - fl;
      const bool in0 = i >= 0 && i < G.N_r, in1 = i + 1 >= 0 && i + 1 < G.N_r;
      if (!in0 && !in1) continue;
      const float *q0 = q + ((size_t)p * G.N_r + (in0 ? i : 0)) * G.N_t;
      const float *q1 = q + ((size_t)p * G.N_r + (in1 ? i + 1 : 0)) * G.N_t;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int tl = lane + 32 * c, t = tb + tl;
        if (tl < TR && t < G.N_t) {
          const float a = in0 ? __ldg(q0 + t) : 0.f, b = in1 ? __ldg(q1 + t) : 0.f;
          acc[c] += (1.f - f) * a + f * b;
        }
      }
    }
    // slice z averages its zovl detector rows z*zovl .. z*zovl + zovl - 1
#pragma unroll
    for (int c = 0; c < 4; c++) rw[lane + 32 * c] = acc[c];
    __syncwarp();
    for (int zl = lane; zl < TR / G.zovl; zl += 32) {
      const int z = tb / G.zovl + zl;
      if (z >= G.N_z) continue;
      float sum = 0.f;
      for (int o = 0; o < G.zovl; o++) sum += rw[zl * G.zovl + o];
      float v = sum * scale;
      if (G.positivity && v < 0.f) v = 0.f;
      xz[z] = v;
    }
    __syncwarp();
  }
}

cudaError_t launch_fbp(const DevGeo &G, const float *y, const float *d, float *q, const float *cosv,
                       const float *sinv, const int *view_idx, const int *view_start, const int *view_num,
                       const int *col_rank, float *x, cudaStream_t st) {
  const size_t smem = ((size_t)G.N_r * (FBP_TT + 1) + (size_t)(G.N_r / 2 + 1)) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute((const void *)k_ramp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 g1((unsigned)G.N_p, (unsigned)((G.N_t + FBP_TT - 1) / FBP_TT));
  k_ramp<<<g1, 256, smem, st>>>(G, y, d, q);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long ncol = (long long)G.N_time * G.N_y * G.N_x;
  k_backproject<<<(unsigned)((ncol + 7) / 8), 256, 0, st>>>(G, q, cosv, sinv, view_idx, view_start, view_num,
                                                             col_rank, x);
  return cudaGetLastError();
}

}  // namespace xtg
