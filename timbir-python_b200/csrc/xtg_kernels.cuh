// xtg_kernels.cuh -- device code of libxtgpu (sm_100a).
//
// Layouts in HBM
//   e, w, y      float [N_p][N_r][N_t]  (reference layout: a column's rows at one
//                                        (view, bin) are contiguous)
//   x            float [N_time][N_y][N_x][N_z]  (z fastest: a column's z-line is
//                                        one contiguous run; the host API keeps
//                                        the reference's [N_time][N_z][N_y][N_x])
//   magmap       float [N_time][nzb][N_y][N_x]
//   work items   int4 {frame, row, col, block}, block = -1 for a whole z-line
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "xt_geom.h"

#define XTG_THREADS 256
#define XTG_AS 4  // A slots per view kept in shared memory (amax <= 4 in the ICD kernel)

struct DevGeo {
  int N_r, N_t, N_p, N_x, N_y, N_z, N_time, zovl, nzb, zstep, amax, positivity;
  float delta_r, delta_t, R0, RMax, x0, y0, delta_xy, OffsetR;
  float MRF_P, C_S, C_T, alpha, Sigma_S_Q, Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P;
  float SF[27];
  float TF, T, delta;
};

// ---------------------------------------------------------------------------
// Exact A-matrix arithmetic.  The reference evaluates `x0 + ((float)k + 0.5) *
// delta` in double (the 0.5 literal is double) and rounds once; float products
// and sums are single roundings with no FMA contraction (gcc, x86-64).  The
// __*_rn intrinsics below are never contracted, so the device reproduces the
// reference's float values bit for bit.
__device__ __forceinline__ float xt_coord(float origin, int idx, float step) {
  return (float)__dadd_rn((double)origin, __dmul_rn(__dadd_rn((double)(float)idx, 0.5), (double)step));
}

// calcAMatrixColumnforAngle (XT_AMatrix.c:50-110) for one (row, col, view).
// The kept bins are contiguous, so they are returned as a dense run
// vals[0..n) starting at bin *first (a bin inside the run that the reference
// drops would get value 0, which contributes nothing either way).
__device__ __forceinline__ int xt_amatrix_view(const DevGeo &G, const float *__restrict__ H, float cp, float sp,
                                               int row, int col, float *vals, int *first) {
  const float x = xt_coord(G.x0, col, G.delta_xy);
  const float y = xt_coord(G.y0, row, G.delta_xy);
  const float r = __fsub_rn(__fmul_rn(x, cp), __fmul_rn(y, sp));
  const float rmin = __fsub_rn(r, G.delta_xy), rmax = __fadd_rn(r, G.delta_xy);
  *first = 0;
  if (rmax < G.R0 || rmin > G.RMax) return 0;
  int imin = (int)floorf(__fdiv_rn(__fsub_rn(rmin, G.R0), G.delta_r));
  int imax = (int)floorf(__fdiv_rn(__fsub_rn(rmax, G.R0), G.delta_r));
  if (imax >= G.N_r) imax = G.N_r - 1;
  if (imin < 0) imin = 0;
  int n = 0, f = -1;
  for (int j = imin; j <= imax; j++) {
    const float rc = xt_coord(G.R0, j, G.delta_r);
    const float dr = fabsf(__fsub_rn(r, rc));
    const int id = (int)floorf(__fdiv_rn(dr, G.OffsetR));
    if (id >= 0 && id < XT_HR_BINS) {
      const float w1 = __fsub_rn(dr, __fmul_rn((float)id, G.OffsetR));
      const float w2 = __fsub_rn(G.OffsetR, w1);
      const float f1 = __fdiv_rn(__fadd_rn(__fmul_rn(w2, H[id]), __fmul_rn(w1, H[id + 1])), G.OffsetR);
      if (f1 > 0.f) {
        if (f < 0) f = j;
        const int s = j - f;
        if (s < XT_AMAX) {
          for (int q = n; q < s; q++) vals[q] = 0.f;  // gap (never seen in practice)
          vals[s] = f1;
          n = s + 1;
        }
      }
    }
  }
  *first = f < 0 ? 0 : f;
  return n;
}

// Register-only form of xt_amatrix_view for at most NS kept bins: slot q holds
// bin imin + q, then leading empty slots are shifted out, so every array
// index is a compile-time constant (no local memory).  Same values as the
// reference's calcAMatrixColumnforAngle.
template <int NS>
__device__ __forceinline__ int xt_amatrix_regs(const DevGeo &G, const float *__restrict__ H, float cp, float sp,
                                               int row, int col, float (&v)[NS], int *first) {
  constexpr int QM = NS + 2;  // imax - imin + 1 never exceeds NS + 2 (floor rounding of +-delta_xy)
  float f[QM];
#pragma unroll
  for (int q = 0; q < QM; q++) f[q] = 0.f;
  *first = 0;
  const float x = xt_coord(G.x0, col, G.delta_xy);
  const float y = xt_coord(G.y0, row, G.delta_xy);
  const float r = __fsub_rn(__fmul_rn(x, cp), __fmul_rn(y, sp));
  const float rmin = __fsub_rn(r, G.delta_xy), rmax = __fadd_rn(r, G.delta_xy);
  int imin = 0;
  if (!(rmax < G.R0 || rmin > G.RMax)) {
    imin = (int)floorf(__fdiv_rn(__fsub_rn(rmin, G.R0), G.delta_r));
    int imax = (int)floorf(__fdiv_rn(__fsub_rn(rmax, G.R0), G.delta_r));
    if (imax >= G.N_r) imax = G.N_r - 1;
    if (imin < 0) imin = 0;
#pragma unroll
    for (int q = 0; q < QM; q++) {
      const int j = imin + q;
      if (j <= imax) {
        const float rc = xt_coord(G.R0, j, G.delta_r);
        const float dr = fabsf(__fsub_rn(r, rc));
        const int id = (int)floorf(__fdiv_rn(dr, G.OffsetR));
        if (id >= 0 && id < XT_HR_BINS) {
          const float w1 = __fsub_rn(dr, __fmul_rn((float)id, G.OffsetR));
          const float w2 = __fsub_rn(G.OffsetR, w1);
          const float f1 = __fdiv_rn(__fadd_rn(__fmul_rn(w2, H[id]), __fmul_rn(w1, H[id + 1])), G.OffsetR);
          if (f1 > 0.f) f[q] = f1;
        }
      }
    }
  }
  // shift leading empty slots out (bounded, constant indices)
  int lead = 0;
#pragma unroll
  for (int it = 0; it < QM - 1; it++) {
    if (f[0] == 0.f && lead < QM - 1) {
#pragma unroll
      for (int q = 0; q < QM - 1; q++) f[q] = f[q + 1];
      f[QM - 1] = 0.f;
      lead++;
    }
  }
  int n = 0;
#pragma unroll
  for (int q = 0; q < QM; q++)
    if (f[q] > 0.f) n = q + 1;
  if (n > NS) n = NS;  // cannot happen: the reference's own buffer holds ceil(3 delta_xy / delta_r) entries
#pragma unroll
  for (int q = 0; q < NS; q++) v[q] = f[q];
  *first = imin + lead;
  return n;
}

// The single entry A[(view, bin), (row, col)], or 0 when the reference keeps
// no entry for that bin.
__device__ __forceinline__ float xt_amatrix_entry(const DevGeo &G, const float *__restrict__ H, float cp, float sp,
                                                  int row, int col, int bin) {
  const float x = xt_coord(G.x0, col, G.delta_xy);
  const float y = xt_coord(G.y0, row, G.delta_xy);
  const float r = __fsub_rn(__fmul_rn(x, cp), __fmul_rn(y, sp));
  const float rmin = __fsub_rn(r, G.delta_xy), rmax = __fadd_rn(r, G.delta_xy);
  if (rmax < G.R0 || rmin > G.RMax) return 0.f;
  int imin = (int)floorf(__fdiv_rn(__fsub_rn(rmin, G.R0), G.delta_r));
  int imax = (int)floorf(__fdiv_rn(__fsub_rn(rmax, G.R0), G.delta_r));
  if (imax >= G.N_r) imax = G.N_r - 1;
  if (imin < 0) imin = 0;
  if (bin < imin || bin > imax) return 0.f;
  const float rc = xt_coord(G.R0, bin, G.delta_r);
  const float dr = fabsf(__fsub_rn(r, rc));
  const int id = (int)floorf(__fdiv_rn(dr, G.OffsetR));
  if (id < 0 || id >= XT_HR_BINS) return 0.f;
  const float w1 = __fsub_rn(dr, __fmul_rn((float)id, G.OffsetR));
  const float w2 = __fsub_rn(G.OffsetR, w1);
  const float f1 = __fdiv_rn(__fadd_rn(__fmul_rn(w2, H[id]), __fmul_rn(w1, H[id + 1])), G.OffsetR);
  return f1 > 0.f ? f1 : 0.f;
}

// ---------------------------------------------------------------------------
// Visiting order.  A balanced 4-round Feistel network on 2h bits with cycle
// walking is a bijection of [0, n); it turns an item counter into a random
// visiting order without a list (the reference draws its order with
// random2(), XT_ICD_update.c:599-631; the order itself is not part of the
// result, the MAP cost is).
__host__ __device__ __forceinline__ uint32_t xt_mix32(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352dU;
  v ^= v >> 15;
  v *= 0x846ca68bU;
  v ^= v >> 16;
  return v;
}

__host__ __device__ __forceinline__ uint32_t xt_perm(uint32_t i, uint32_t n, uint64_t key) {
  int h = 1;
  while ((1ull << (2 * h)) < (unsigned long long)n) h++;
  const uint32_t mask = (1u << h) - 1u;
  uint32_t v = i;
  do {  // terminates: the walk stays on i's cycle of a permutation of [0, 4^h)
    uint32_t L = v >> h, R = v & mask;
    for (int k = 0; k < 4; k++) {
      const uint32_t F = xt_mix32(R ^ (uint32_t)key ^ (uint32_t)(key >> 32) * 0x9E3779B9u ^ (uint32_t)k * 0x85ebca6bu) & mask;
      const uint32_t nl = R;
      R = L ^ F;
      L = nl;
    }
    v = (L << h) | R;
  } while (v >= n);
  return v;
}

// ---------------------------------------------------------------------------
// qGGMRF surrogate coefficient b = filter * rho'(delta)/delta (CE_QGGMRF_*,
// XT_ICD_update.c:79-125) with q = 2: rho'(d)/d = (q - (q-p) t1/t3)/(t3 sigma_q),
// t1 = |d|^(q-p)/sigma_qp, t3 = c + t1; at d = 0 the limit q/(sigma_q c).
__device__ __forceinline__ float xt_qggmrf_coef(float d, float sq, float sqp, float c, float p) {
  if (d == 0.f) return 2.0f / (sq * c);
  const float t1 = powf(fabsf(d), 2.0f - p) / sqp;
  const float t3 = c + t1;
  return (2.0f - (2.0f - p) * t1 / t3) / (t3 * sq);
}

// red.global.add on four consecutive floats: no lost updates when two
// columns in flight share sinogram entries.
__device__ __forceinline__ void xt_red_add4(float *p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

__device__ __forceinline__ uint32_t xt_f2key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float xt_key2f(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
