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

// ------------------------------------------------ bin-major A table ------
// The A entries regrouped by sinogram row (view p, detector bin r): row
// (p, r) lists (column j N_x + k, A) for every column of p's frame that
// reaches bin r, in increasing (j, k) -- the order in which the reference
// adds a column's contribution to that entry (initErrorSinogam,
// XT_ICD_update.c:551-569).  Built once per context by the enumeration of
// k_fp_bins, so every value is the exact A of calcAMatrixColumnforAngle
// (XT_AMatrix.c:50-110).  Lane b of a warp owns bin rb + b of the warp's 32
// bins: for each hit column the lanes test their own bin in parallel, so the
// appends of a bin stay in column order without atomics.
template <int FILL, int NS>
__global__ void __launch_bounds__(FP_WARPS * 32) k_csr_build(DevGeo G, CsrBuildArgs B) {
  extern __shared__ __align__(16) unsigned char cb_sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float *vsm = reinterpret_cast<float *>(cb_sm) + (size_t)warp * 32 * NS;
  const int p = blockIdx.x;
  const int rb = (blockIdx.y * FP_WARPS + warp) * 32;
  if (rb >= G.N_r) return;  // whole warp; no block-wide barrier follows
  const float cp = B.cosv[p], sp = B.sinv[p];
  const float *H = B.hr + (size_t)p * XT_HR_STRIDE;
  const double lo = (double)G.R0 + (double)rb * G.delta_r - G.delta_xy - B.win_margin;
  const double hi = (double)G.R0 + (double)(rb + 32) * G.delta_r + G.delta_xy + B.win_margin;
  const int r = rb + lane;
  const bool own = r < G.N_r;
  long long cur = 0;
  int cnt = 0;
  if (FILL && own) cur = B.ptr[(size_t)p * G.N_r + r];
  for (int j = 0; j < G.N_y; j++) {
    int klo, khi;
    if (!fp_col_range(G, cp, sp, xt_coord(G.y0, j, G.delta_xy), lo, hi, &klo, &khi)) continue;
    for (int kb = klo; kb <= khi; kb += 32) {
      const int k = kb + lane;
      float v[NS];
#pragma unroll
      for (int q = 0; q < NS; q++) v[q] = 0.f;
      int first = 0, n = 0;
      if (k <= khi) n = xt_amatrix_regs<NS>(G, H, cp, sp, j, k, v, &first);
      const int slo = max(0, rb - first), shi = min(n, rb + 32 - first);
      const unsigned hit = __ballot_sync(0xffffffffu, slo < shi);
      if (!hit) continue;
#pragma unroll
      for (int q = 0; q < NS; q++) vsm[lane * NS + q] = v[q];
      const int pk = (int)(((unsigned)(first - rb + 64) << 16) | ((unsigned)slo << 8) | (unsigned)shi);
      __syncwarp();
      unsigned mk = hit;
      while (mk) {
        const int l = __ffs(mk) - 1;
        mk &= mk - 1;
        const int q = __shfl_sync(0xffffffffu, pk, l);
        const int sl = (q >> 8) & 0xFF, sh = q & 0xFF;
        const int sidx = lane - ((q >> 16) - 64);  // this lane's bin within the column's run
        if (own && sidx >= sl && sidx < sh) {
          const float a = vsm[l * NS + sidx];
          if (a != 0.f) {
            if (FILL) {
              B.ent[cur] = make_int2((j * G.N_x + kb + l) * G.N_z, __float_as_int(a));
              cur++;
            } else {
              cnt++;
            }
          }
        }
      }
      __syncwarp();  // the staged entries are rewritten by the next round
    }
  }
  if (!FILL && own) B.count[(size_t)p * G.N_r + r] = cnt;
}

template <int FILL>
static cudaError_t launch_csr_build_t(const DevGeo &G, const CsrBuildArgs &B, int ns, cudaStream_t st) {
  const int nsv = ns <= 3 ? 3 : ns <= 4 ? 4 : 12;
  const size_t smem = (size_t)FP_WARPS * 32 * nsv * sizeof(float);
  dim3 grid((unsigned)G.N_p, (unsigned)((G.N_r + FP_WARPS * 32 - 1) / (FP_WARPS * 32)));
  if (ns <= 3)
    k_csr_build<FILL, 3><<<grid, FP_WARPS * 32, smem, st>>>(G, B);
  else if (ns <= 4)
    k_csr_build<FILL, 4><<<grid, FP_WARPS * 32, smem, st>>>(G, B);
  else
    k_csr_build<FILL, 12><<<grid, FP_WARPS * 32, smem, st>>>(G, B);
  return cudaGetLastError();
}

cudaError_t launch_csr_build(const DevGeo &G, const CsrBuildArgs &B, int fill, int ns, cudaStream_t st) {
  return fill ? launch_csr_build_t<1>(G, B, ns, st) : launch_csr_build_t<0>(G, B, ns, st);
}

// Forward projection from the bin-major table: one warp per sinogram row
// (view, bin) and 64 detector rows.  Every lane reads each entry
// {z-line offset, A} (a broadcast from L1; two entries per 16-byte load) and
// its rows of that z-line (PAIR: rows 2 lane, 2 lane + 1 as one 8-byte load
// when a slice covers one detector row; the warp's loads form one 256-byte
// run), and accumulates in registers, entries in table order: in FP32
// (__fadd_rn(__fmul_rn)) that is the reference's summation order, so MODE
// 0 / 1 are bit-identical to k_fp_bins and to initErrorSinogam; MODE 2 / 3
// accumulate in FP64 in the same order (a product of two FP32 values is
// exact in FP64, so the sums equal k_fp_bins' bit for bit).  Eight entries
// are loaded before any is added.  The eight warps of a CTA take eight
// consecutive bins of one view, which share most of their columns, so many
// z-lines are L1 hits.  FULL: every 64-row chunk is complete (N_t a multiple
// of 64), so no lane needs a bounds test.
#define CSR_WARPS 8
template <int MODE, typename ACC, bool PAIR, bool FULL>
__global__ void __launch_bounds__(CSR_WARPS * 32) k_fp_csr(DevGeo G, FpArgs F, CsrView T) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int p = blockIdx.x;
  const int r = blockIdx.y * CSR_WARPS + warp;
  if (r >= G.N_r) return;  // whole warp; no block-wide barrier follows
  const int t0 = blockIdx.z * 64, nt = FULL ? 64 : min(64, G.N_t - t0);
  // rows of this lane: PAIR (zovl == 1, N_t even): 2 lane, 2 lane + 1, one
  // float2 at slice t0 + 2 lane; otherwise lane and lane + 32
  const int ta = PAIR ? 2 * lane : lane, tb = PAIR ? 2 * lane + 1 : lane + 32;
  const bool va = FULL || ta < nt, vb = FULL || tb < nt;
  const float *xf = F.x + (size_t)F.fov[p] * G.N_y * G.N_x * G.N_z;
  const float *xla = xf + (t0 + ta) / G.zovl, *xlb = xf + (t0 + tb) / G.zovl;
  const long long e0 = T.ptr[(size_t)p * G.N_r + r], e1 = T.ptr[(size_t)p * G.N_r + r + 1];
  ACC acc_a = (ACC)0, acc_b = (ACC)0;
  auto add = [&](float xa, float xb, float a) {
    if (MODE <= 1) {
      acc_a = __fadd_rn(acc_a, __fmul_rn(xa, a));
      acc_b = __fadd_rn(acc_b, __fmul_rn(xb, a));
    } else {
      acc_a += (ACC)xa * (ACC)a;
      acc_b += (ACC)xb * (ACC)a;
    }
  };
  auto load = [&](int off, float &xa, float &xb) {
    if (PAIR) {
      const float2 v = va ? __ldg(reinterpret_cast<const float2 *>(xla + off)) : make_float2(0.f, 0.f);
      xa = v.x;
      xb = v.y;
    } else {
      xa = va ? __ldg(xla + off) : 0.f;
      xb = vb ? __ldg(xlb + off) : 0.f;
    }
  };
  long long i = e0;
  if (i < e1 && (i & 1)) {  // to a 16-byte boundary of the entry array
    const int2 en = __ldg(T.ent + i);
    float xa, xb;
    load(en.x, xa, xb);
    add(xa, xb, __int_as_float(en.y));
    i++;
  }
  for (; i + 8 <= e1; i += 8) {
    const int4 *q = reinterpret_cast<const int4 *>(T.ent + i);
    int4 qv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) qv[u] = __ldg(q + u);
    float xa[8], xb[8];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      load(qv[u].x, xa[2 * u], xb[2 * u]);
      load(qv[u].z, xa[2 * u + 1], xb[2 * u + 1]);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      add(xa[2 * u], xb[2 * u], __int_as_float(qv[u].y));
      add(xa[2 * u + 1], xb[2 * u + 1], __int_as_float(qv[u].w));
    }
  }
  for (; i < e1; i++) {
    const int2 en = __ldg(T.ent + i);
    float xa, xb;
    load(en.x, xa, xb);
    add(xa, xb, __int_as_float(en.y));
  }
  double cacc = 0.0;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int t = h ? tb : ta;
    if (!FULL && t >= nt) continue;
    const ACC sacc = h ? acc_b : acc_a;
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
  if (MODE >= 2) {
    for (int off = 16; off > 0; off >>= 1) cacc += __shfl_xor_sync(0xffffffffu, cacc, off);
    if (lane == 0) atomicAdd(&F.cost_slots[(blockIdx.x * 7 + r + blockIdx.z) % 64], cacc);
  }
}

template <bool PAIR, bool FULL>
static void launch_fp_csr_t(const DevGeo &G, const FpArgs &F, const CsrView &T, int mode, cudaStream_t st) {
  dim3 grid((unsigned)G.N_p, (unsigned)((G.N_r + CSR_WARPS - 1) / CSR_WARPS), (unsigned)((G.N_t + 63) / 64));
  switch (mode) {
    case 0: k_fp_csr<0, float, PAIR, FULL><<<grid, CSR_WARPS * 32, 0, st>>>(G, F, T); break;
    case 1: k_fp_csr<1, float, PAIR, FULL><<<grid, CSR_WARPS * 32, 0, st>>>(G, F, T); break;
    case 2: k_fp_csr<2, double, PAIR, FULL><<<grid, CSR_WARPS * 32, 0, st>>>(G, F, T); break;
    default: k_fp_csr<3, double, PAIR, FULL><<<grid, CSR_WARPS * 32, 0, st>>>(G, F, T); break;
  }
}

cudaError_t launch_fp_csr(const DevGeo &G, const FpArgs &F, const CsrView &T, int mode, cudaStream_t st) {
  // paired rows need one detector row per slice, an even row count (so a
  // chunk never ends inside a pair) and 8-byte aligned z-lines
  if (G.zovl == 1 && G.N_t % 2 == 0 && G.N_z % 2 == 0) {
    if (G.N_t % 64 == 0)
      launch_fp_csr_t<true, true>(G, F, T, mode, st);
    else
      launch_fp_csr_t<true, false>(G, F, T, mode, st);
  } else {
    launch_fp_csr_t<false, false>(G, F, T, mode, st);
  }
  return cudaGetLastError();
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
