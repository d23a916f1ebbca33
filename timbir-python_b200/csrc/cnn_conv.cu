// cnn_conv.cu -- 3x3x3 convolutions of the warm-start network as implicit
// GEMMs on the tcgen05 tensor cores (BF16 in, FP32 accumulation in TMEM).
//
// Activations are channels-last volumes [nb][Y][X][Z][C] (C a multiple of 8,
// so 8 channels are one 16-byte load), padding 1, stride 1.  Weights of a
// layer with cin inputs and cout outputs are stored K-major as
// W[cout][kpad], k = tap*cin + ci, tap = (dy+1)*9 + (dx+1)*3 + (dz+1),
// kpad = 27*cin rounded up to 64 (zero tail).
//
//   forward  out[v][co] = act(bias[co] + sum_{tap,ci} in[v + d(tap)][ci] W[co][tap][ci])
//            GEMM M = voxels, N = cout, K = 27 cin; A gathered (K-major), B = W.
//   dgrad    din[u][ci] = sum_{tap,co} dout[u - d(tap)][co] W[co][tap][ci]
//            the same kernel with the offsets negated and B = Wt[ci][tap][co].
//   wgrad    dW[tap][ci][co] += sum_v in[v + d(tap)][ci] dout[v][co]
//            GEMM M = 27 cin, N = cout, K = voxels (split over CTAs, FP32
//            atomics into dW); operands transposed to K-major while staged.
#include <cuda_bf16.h>

#include "cnn_tc.cuh"
#include "xtg_cnn_internal.h"

namespace xtc {

#define CONV_THREADS 128
#define KT 64  // K elements per stage

__device__ __forceinline__ void tap_offset(int tap, int &dy, int &dx, int &dz) {
  dy = tap / 9 - 1;
  dx = (tap / 3) % 3 - 1;
  dz = tap % 3 - 1;
}

// Block-uniform bounded wait; on timeout sets *err and returns false.
__device__ __forceinline__ bool wait_stage(uint64_t *mbar, uint32_t parity, int *err, long long limit = 1ll << 24) {
  const bool ok = mbar_wait(mbar, parity, limit);
  const bool all = __syncthreads_and(ok) != 0;
  if (!all && threadIdx.x == 0) atomicExch(err, 1);
  return all;
}

// EPI: 0 = bias + ReLU -> bf16, 1 = plain -> bf16, 2 = plain -> fp32
template <int SIGN, int EPI>
__global__ void __launch_bounds__(CONV_THREADS) k_conv_tc(ConvShape s, const __nv_bfloat16 *__restrict__ in,
                                                          const __nv_bfloat16 *__restrict__ w,
                                                          const float *__restrict__ bias, void *out, int *err) {
  extern __shared__ __align__(128) uint8_t sm[];
  const int N = s.n;
  uint8_t *sA = sm;                              // [2][KT/8][128][16 B]
  uint8_t *sB = sm + 2 * 128 * KT * 2;           // [2][KT/8][N][16 B]
  const uint32_t A_STAGE = 128 * KT * 2, B_STAGE = (uint32_t)N * KT * 2;
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long M = (long long)s.nb * s.Y * s.X * s.Z;
  const long long mv = (long long)blockIdx.x * 128 + tid;  // this thread's output voxel (A row)
  const bool mval = mv < M;
  int b = 0, yy = 0, xx = 0, zz = 0;
  if (mval) {
    long long r = mv;
    zz = (int)(r % s.Z);
    r /= s.Z;
    xx = (int)(r % s.X);
    r /= s.X;
    yy = (int)(r % s.Y);
    b = (int)(r / s.Y);
  }
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(&tbase, tmem_cols(N));
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  const uint32_t idesc = idesc_bf16(N, 0, 0);
  const int nk = s.kpad / KT;
  bool ok = true;
  for (int kt = 0; kt < nk && ok; kt++) {
    const int st = kt & 1;
    if (kt >= 2) ok = wait_stage(&mbar[st], (uint32_t)((kt - 2) >> 1) & 1u, err);
    if (!ok) break;
    // A: this thread's row, 8 chunks of 8 K elements (one tap, 8 channels each)
    uint8_t *a = sA + st * A_STAGE;
    // (tap, channel) of the stage's first chunk; the next chunks step 8
    // channels (cin is a multiple of 8), so one division per stage
    int tap = (kt * KT) / s.cin, ci = kt * KT - tap * s.cin;
#pragma unroll
    for (int c = 0; c < KT / 8; c++, ci += 8) {
      if (ci >= s.cin) {
        ci -= s.cin;
        tap++;
      }
      int4 v = make_int4(0, 0, 0, 0);
      if (mval && tap < 27) {
        int dy, dx, dz;
        tap_offset(tap, dy, dx, dz);
        const int y2 = yy + SIGN * dy, x2 = xx + SIGN * dx, z2 = zz + SIGN * dz;
        if (y2 >= 0 && y2 < s.Y && x2 >= 0 && x2 < s.X && z2 >= 0 && z2 < s.Z)
          v = __ldg(reinterpret_cast<const int4 *>(in + ((((size_t)b * s.Y + y2) * s.X + x2) * s.Z + z2) * s.cin + ci));
      }
      *reinterpret_cast<int4 *>(a + c * (128 * 16) + tid * 16) = v;
    }
    // B: N rows x 8 chunks of the weight matrix
    uint8_t *bb = sB + st * B_STAGE;
    for (int i = tid; i < N * (KT / 8); i += CONV_THREADS) {
      const int c = i / N, n = i - c * N;
      const int4 v = __ldg(reinterpret_cast<const int4 *>(w + (size_t)n * s.kpad + kt * KT + c * 8));
      *reinterpret_cast<int4 *>(bb + c * (N * 16) + n * 16) = v;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(a), b0 = smem_u32(bb);
#pragma unroll
      for (int ks = 0; ks < KT / 16; ks++) {
        const uint64_t da = sdesc(a0 + ks * 2 * 128 * 16, 128 * 16, 128);
        const uint64_t db = sdesc(b0 + ks * 2 * N * 16, N * 16, 128);
        mma_bf16(tmem, da, db, idesc, (kt > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&mbar[st]);
    }
  }
  if (ok) {
    const int last = nk - 1;
    ok = wait_stage(&mbar[last & 1], (uint32_t)(last >> 1) & 1u, err);
  }
  tc_fence_after();
  if (ok) {
    // epilogue: warp w holds accumulator rows 32w .. 32w+31 (TMEM lanes)
    for (int n0 = 0; n0 < N; n0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      if (!mval) continue;
      if (EPI == 2) {
        float *o = reinterpret_cast<float *>(out) + (size_t)mv * N + n0;
#pragma unroll
        for (int q = 0; q < 16; q += 4) *reinterpret_cast<float4 *>(o + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
      } else {
        __align__(16) __nv_bfloat16 h[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          float t = v[q];
          if (EPI == 0) t = fmaxf(t + bias[n0 + q], 0.f);
          h[q] = __float2bfloat16_rn(t);
        }
        __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(out) + (size_t)mv * N + n0;
        *reinterpret_cast<int4 *>(o) = *reinterpret_cast<const int4 *>(h);
        *reinterpret_cast<int4 *>(o + 8) = *reinterpret_cast<const int4 *>(h + 8);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, tmem_cols(N));
  }
}

// 8x8 transpose of BF16: row v of the input is voxel v's 8 channels (one int4);
// row c of the output holds channel c of the 8 voxels
__device__ __forceinline__ void transpose8(const int4 (&in)[8], int4 (&out)[8]) {
  const uint32_t *a = reinterpret_cast<const uint32_t *>(in);
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const uint32_t sel = (c & 1) ? 0x7632u : 0x5410u;
    uint32_t o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] = __byte_perm(a[(2 * q) * 4 + c / 2], a[(2 * q + 1) * 4 + c / 2], sel);
    out[c] = make_int4((int)o[0], (int)o[1], (int)o[2], (int)o[3]);
  }
}

// decode a voxel index into (batch, y, x, z)
__device__ __forceinline__ void voxel_coords(const ConvShape &s, long long v, int &b, int &yy, int &xx, int &zz) {
  zz = (int)(v % s.Z);
  v /= s.Z;
  xx = (int)(v % s.X);
  v /= s.X;
  yy = (int)(v % s.Y);
  b = (int)(v / s.Y);
}

// wgrad: M = 27*cin rows (tap, ci), N = cout, K = voxels [k0, k0 + kchunk).
// Both operands are staged K-major (voxels contiguous): each thread loads the
// 8-channel rows of 8 consecutive voxels and transposes them in registers.
__global__ void __launch_bounds__(CONV_THREADS) k_wgrad_tc(ConvShape s, const __nv_bfloat16 *__restrict__ in,
                                                           const __nv_bfloat16 *__restrict__ dout, float *dw,
                                                           int kchunk, int *err) {
  extern __shared__ __align__(128) uint8_t sm[];
  const int N = s.n;
  uint8_t *sA = sm;
  uint8_t *sB = sm + 2 * 128 * KT * 2;
  const uint32_t A_STAGE = 128 * KT * 2, B_STAGE = (uint32_t)N * KT * 2;
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long Mv = (long long)s.nb * s.Y * s.X * s.Z;
  const int rows = 27 * s.cin;
  const int r0 = blockIdx.x * 128;
  const long long k0 = (long long)blockIdx.y * kchunk;
  const long long kend = k0 + kchunk < Mv ? k0 + kchunk : Mv;
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(&tbase, tmem_cols(N));
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  const uint32_t idesc = idesc_bf16(N, 0, 0);
  const int nk = (int)((kend - k0 + KT - 1) / KT);
  // this thread's A unit: row group ga (8 rows of one tap) x voxel chunk ca
  const int ga = tid >> 3, ca = tid & 7;
  const int ra = r0 + ga * 8;
  int tap = 0, ci = 0, ddy = 0, ddx = 0, ddz = 0;
  if (ra < rows) {
    tap = ra / s.cin;
    ci = ra - tap * s.cin;
    tap_offset(tap, ddy, ddx, ddz);
  }
  bool ok = nk > 0;
  for (int kt = 0; kt < nk && ok; kt++) {
    const int st = kt & 1;
    if (kt >= 2) ok = wait_stage(&mbar[st], (uint32_t)((kt - 2) >> 1) & 1u, err);
    if (!ok) break;
    const long long vb = k0 + (long long)kt * KT;
    uint8_t *a = sA + st * A_STAGE;
    {
      int4 ld[8], tr[8];
      if (s.Z % 8 == 0) {
        // the 8 voxels start at a multiple of 8 and lie on one z-line: one
        // coordinate decode for the group
        const long long v0 = vb + ca * 8;
        int b = 0, yy = 0, xx = 0, zz = 0;
        if (v0 < kend) voxel_coords(s, v0, b, yy, xx, zz);
        const int y2 = yy + ddy, x2 = xx + ddx;
        const bool line = ra < rows && y2 >= 0 && y2 < s.Y && x2 >= 0 && x2 < s.X;
        const __nv_bfloat16 *base = line ? in + (((size_t)b * s.Y + y2) * s.X + x2) * s.Z * s.cin + ci : in;
#pragma unroll
        for (int u = 0; u < 8; u++) {
          ld[u] = make_int4(0, 0, 0, 0);
          const int z2 = zz + u + ddz;
          if (line && v0 + u < kend && z2 >= 0 && z2 < s.Z)
            ld[u] = __ldg(reinterpret_cast<const int4 *>(base + (size_t)z2 * s.cin));
        }
      } else {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          ld[u] = make_int4(0, 0, 0, 0);
          const long long v = vb + ca * 8 + u;
          if (ra < rows && v < kend) {
            int b, yy, xx, zz;
            voxel_coords(s, v, b, yy, xx, zz);
            const int y2 = yy + ddy, x2 = xx + ddx, z2 = zz + ddz;
            if (y2 >= 0 && y2 < s.Y && x2 >= 0 && x2 < s.X && z2 >= 0 && z2 < s.Z)
              ld[u] = __ldg(reinterpret_cast<const int4 *>(
                  in + ((((size_t)b * s.Y + y2) * s.X + x2) * s.Z + z2) * s.cin + ci));
          }
        }
      }
      transpose8(ld, tr);
#pragma unroll
      for (int c = 0; c < 8; c++) *reinterpret_cast<int4 *>(a + ca * (128 * 16) + (ga * 8 + c) * 16) = tr[c];
    }
    uint8_t *bb = sB + st * B_STAGE;
    for (int unit = tid; unit < (N / 8) * 8; unit += CONV_THREADS) {
      const int g = unit >> 3, cb = unit & 7;
      int4 ld[8], tr[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const long long v = vb + cb * 8 + u;
        ld[u] = (v < kend) ? __ldg(reinterpret_cast<const int4 *>(dout + (size_t)v * N + g * 8)) : make_int4(0, 0, 0, 0);
      }
      transpose8(ld, tr);
#pragma unroll
      for (int c = 0; c < 8; c++) *reinterpret_cast<int4 *>(bb + cb * (N * 16) + (g * 8 + c) * 16) = tr[c];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(a), b0 = smem_u32(bb);
#pragma unroll
      for (int ks = 0; ks < KT / 16; ks++) {
        const uint64_t da = sdesc(a0 + ks * 2 * 128 * 16, 128 * 16, 128);
        const uint64_t db = sdesc(b0 + ks * 2 * N * 16, N * 16, 128);
        mma_bf16(tmem, da, db, idesc, (kt > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&mbar[st]);
    }
  }
  if (ok) {
    const int last = nk - 1;
    ok = wait_stage(&mbar[last & 1], (uint32_t)(last >> 1) & 1u, err);
  }
  tc_fence_after();
  if (ok) {
    const int r = r0 + tid;
    for (int n0 = 0; n0 < N; n0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      if (r < rows) {
#pragma unroll
        for (int q = 0; q < 16; q++) atomicAdd(dw + (size_t)r * N + n0 + q, v[q]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, tmem_cols(N));
  }
}

// The network's first layer: two input channels (the FBP image and the start
// image, FP32 [nb][Y][X][Z], times scale), so K = 27 taps x 2 = 54, padded to
// 64: one MMA stage whose A rows are gathered straight from the FP32 volumes
// (the input packing fused into the convolution).  w64: [n][64] BF16,
// k = 2 tap + channel.  Output: ReLU(acc + bias) in BF16 [voxel][n].
__global__ void __launch_bounds__(CONV_THREADS) k_conv_first(int nb, int Y, int X, int Z, const float *__restrict__ fa,
                                                             const float *__restrict__ fb, float scale,
                                                             const __nv_bfloat16 *__restrict__ w64,
                                                             const float *__restrict__ bias, int N,
                                                             __nv_bfloat16 *__restrict__ out, int *err) {
  extern __shared__ __align__(128) uint8_t sm[];
  uint8_t *sA = sm;                 // [8][128][16 B]
  uint8_t *sB = sm + 128 * 64 * 2;  // [8][N][16 B]
  __shared__ uint64_t mbar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long M = (long long)nb * Y * X * Z;
  const long long mv = (long long)blockIdx.x * 128 + tid;
  const bool mval = mv < M;
  int b = 0, yy = 0, xx = 0, zz = 0;
  if (mval) {
    long long r = mv;
    zz = (int)(r % Z);
    r /= Z;
    xx = (int)(r % X);
    r /= X;
    yy = (int)(r % Y);
    b = (int)(r / Y);
  }
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(&tbase, tmem_cols(N));
  // A: this thread's voxel, K = (tap, channel)
  __align__(16) __nv_bfloat16 row[64];
#pragma unroll
  for (int t = 0; t < 27; t++) {
    int dy, dx, dz;
    tap_offset(t, dy, dx, dz);
    const int y2 = yy + dy, x2 = xx + dx, z2 = zz + dz;
    float va = 0.f, vb = 0.f;
    if (mval && y2 >= 0 && y2 < Y && x2 >= 0 && x2 < X && z2 >= 0 && z2 < Z) {
      const size_t o = (((size_t)b * Y + y2) * X + x2) * Z + z2;
      va = __ldg(fa + o) * scale;
      vb = __ldg(fb + o) * scale;
    }
    row[2 * t] = __float2bfloat16_rn(va);
    row[2 * t + 1] = __float2bfloat16_rn(vb);
  }
#pragma unroll
  for (int k = 54; k < 64; k++) row[k] = __float2bfloat16_rn(0.f);
#pragma unroll
  for (int c = 0; c < 8; c++)
    *reinterpret_cast<int4 *>(sA + c * (128 * 16) + tid * 16) = *reinterpret_cast<const int4 *>(row + 8 * c);
  for (int i = tid; i < N * 8; i += CONV_THREADS) {
    const int c = i / N, n = i - c * N;
    *reinterpret_cast<int4 *>(sB + c * (N * 16) + n * 16) =
        __ldg(reinterpret_cast<const int4 *>(w64 + (size_t)n * 64 + c * 8));
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(N, 0, 0), a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
    for (int ks = 0; ks < 4; ks++)
      mma_bf16(tmem, sdesc(a0 + ks * 2 * 128 * 16, 128 * 16, 128), sdesc(b0 + ks * 2 * N * 16, N * 16, 128), idesc,
               ks > 0 ? 1u : 0u);
    mma_commit(&mbar);
  }
  const bool ok = wait_stage(&mbar, 0, err);
  tc_fence_after();
  if (ok) {
    for (int n0 = 0; n0 < N; n0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      if (!mval) continue;
      __align__(16) __nv_bfloat16 h[16];
#pragma unroll
      for (int q = 0; q < 16; q++) h[q] = __float2bfloat16_rn(fmaxf(v[q] + bias[n0 + q], 0.f));
      __nv_bfloat16 *o = out + (size_t)mv * N + n0;
      *reinterpret_cast<int4 *>(o) = *reinterpret_cast<const int4 *>(h);
      *reinterpret_cast<int4 *>(o + 8) = *reinterpret_cast<const int4 *>(h + 8);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, tmem_cols(N));
  }
}

// [n][kpad] with k = tap * cin + ci (ci < 2 real) -> [n][64] with k = 2 tap + ci
__global__ void k_pack_first(int n, int cin, int kpad, const __nv_bfloat16 *__restrict__ w,
                             __nv_bfloat16 *__restrict__ w64) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * 64) return;
  const int nn = i / 64, k = i % 64;
  w64[i] = k < 54 ? w[(size_t)nn * kpad + (k / 2) * cin + (k % 2)] : __float2bfloat16_rn(0.f);
}

// Dynamic shared memory per CTA: the two operand stages, raised where needed
// so that no more CTAs fit on an SM (228 KB) than its 512 TMEM columns hold.
static size_t conv_smem(int n) {
  const size_t need = (size_t)2 * 128 * KT * 2 + (size_t)2 * n * KT * 2;
  const size_t per_sm = 228 * 1024;
  const size_t fit = 512 / xtc::tmem_cols(n);  // CTAs whose accumulators fit at once
  const size_t floor_bytes = per_sm / (fit + 1) + 1024;
  return need > floor_bytes ? need : floor_bytes;
}

cudaError_t conv_forward(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                         void *out, int epi, int sign, int *err, cudaStream_t st) {
  if (s.n % 16 || s.n < 16 || s.n > 256 || s.cin % 8 || s.kpad % KT || s.kpad < 27 * s.cin) return cudaErrorInvalidValue;
  const long long M = (long long)s.nb * s.Y * s.X * s.Z;
  const size_t smem = conv_smem(s.n);
  typedef void (*K)(ConvShape, const __nv_bfloat16 *, const __nv_bfloat16 *, const float *, void *, int *);
  K k;
  if (sign > 0)
    k = epi == 0 ? k_conv_tc<1, 0> : epi == 1 ? k_conv_tc<1, 1> : k_conv_tc<1, 2>;
  else
    k = epi == 0 ? k_conv_tc<-1, 0> : epi == 1 ? k_conv_tc<-1, 1> : k_conv_tc<-1, 2>;
  cudaError_t e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<(unsigned)((M + 127) / 128), CONV_THREADS, smem, st>>>(s, in, w, bias, out, err);
  return cudaGetLastError();
}

cudaError_t conv_wgrad(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, float *dw, int *err,
                       cudaStream_t st, int path) {
  if (s.n % 16 || s.n < 16 || s.n > 256 || s.cin % 8) return cudaErrorInvalidValue;
  if (path != 1 && wgrad_tile_supported(s)) {
    const cudaError_t e = conv_wgrad_tile(s, in, dout, dw, err, st);
    if (e != cudaErrorNotSupported || path == 2) return e;
  } else if (path == 2) {
    return cudaErrorNotSupported;
  }
  const long long M = (long long)s.nb * s.Y * s.X * s.Z;
  const int mt = (27 * s.cin + 127) / 128;
  // enough K splits to fill the GPU twice over, each a multiple of KT voxels
  long long splits = (2 * 148 + mt - 1) / mt;
  if (splits < 1) splits = 1;
  long long kchunk = (M + splits - 1) / splits;
  kchunk = (kchunk + KT - 1) / KT * KT;
  splits = (M + kchunk - 1) / kchunk;
  const size_t smem = conv_smem(s.n);
  cudaError_t e = cudaFuncSetAttribute((const void *)k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_wgrad_tc<<<dim3((unsigned)mt, (unsigned)splits), CONV_THREADS, smem, st>>>(s, in, dout, dw, (int)kchunk, err);
  return cudaGetLastError();
}

}  // namespace xtc

namespace xtc {

cudaError_t conv_first_pack(int n, int cin, int kpad, const __nv_bfloat16 *w, __nv_bfloat16 *w64, cudaStream_t st) {
  if (cin < 2) return cudaErrorInvalidValue;
  k_pack_first<<<(n * 64 + 255) / 256, 256, 0, st>>>(n, cin, kpad, w, w64);
  return cudaGetLastError();
}

cudaError_t conv_first(int nb, int Y, int X, int Z, const float *a, const float *b, float scale,
                       const __nv_bfloat16 *w64, const float *bias, int n, __nv_bfloat16 *out, int *err,
                       cudaStream_t st) {
  if (n % 16 || n < 16 || n > 256) return cudaErrorInvalidValue;
  const long long M = (long long)nb * Y * X * Z;
  size_t smem = (size_t)128 * 64 * 2 + (size_t)n * 64 * 2;
  // no more CTAs on an SM than its 512 TMEM columns hold
  const size_t fit = 512 / tmem_cols(n), floor_bytes = 228 * 1024 / (fit + 1) + 1024;
  if (smem < floor_bytes) smem = floor_bytes;
  cudaError_t e =
      cudaFuncSetAttribute((const void *)k_conv_first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_conv_first<<<(unsigned)((M + 127) / 128), CONV_THREADS, smem, st>>>(nb, Y, X, Z, a, b, scale, w64, bias, n, out,
                                                                         err);
  return cudaGetLastError();
}

// The bounded-wait path of the tensor-core kernels exercised alone: one CTA
// waits on a fresh mbarrier (count 1) with `limit` polls, after thread 0
// has arrived on it or not.  Nothing is in flight, so a wait that gives up
// leaves nothing behind; it sets *err like a convolution's would.
__global__ void k_wait_selftest(int arrive, long long limit, int *err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
  wait_stage(&bar, 0, err, limit);
}

cudaError_t wait_selftest(int arrive, long long limit, int *err, cudaStream_t st) {
  k_wait_selftest<<<1, 128, 0, st>>>(arrive, limit, err);
  return cudaGetLastError();
}

}  // namespace xtc
