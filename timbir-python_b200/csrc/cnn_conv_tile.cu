// cnn_conv_tile.cu -- 3x3x3 convolutions of the warm-start network on tiles
// staged once by TMA (BF16 in, FP32 accumulation in TMEM).
//
// The gather kernel in cnn_conv.cu builds every A row (voxel x 64 K values)
// with per-thread loads: each input voxel is fetched 27 times.  Here a CTA
// owns an output tile of 128 x-voxels x TZ z-lines of one y-row; one TMA box
// per 16-channel chunk stages the tile's input halo (130 x (TZ + 2) x 3
// voxels, zero filled outside the volume) in shared memory once, one 32-byte
// row per voxel (16 channels, the 32-byte swizzle), x fastest:
// row r = (y' * TZS + z') * TXS + x'.  In that layout the A operand of tap
// (dy, dx, dz) for output line z is the run of 128 rows starting at
// r0(z) + (dy * TZS + dz) * TXS + dx -- one shared-memory descriptor with a
// shifted start address.  No im2col gather is ever materialised.
//
// One MMA serves up to three output lines: staged z-line L feeds output lines
// L - 1, L and L + 1 through the taps dz = +1, 0, -1, so with the weights of
// those three taps stacked along N (the accumulators of consecutive output
// lines are consecutive TMEM columns) each (L, dy, dx) is one MMA of N = up to
// 3 cout -- half the MMAs, and half the A reads from shared memory, of one
// MMA per (output line, tap).  The accumulators are zeroed by the epilogue
// warps (tcgen05.st) and every MMA accumulates.
//
// Weights come pre-packed per 16-channel chunk as
// Wp[chunk][dy, dx][half][dz = +1, 0, -1][n][8] (offsets as the kernel applies
// them, i.e. mirrored for sign -1) and are copied with one bulk copy per stage.  One thread issues the TMA, the bulk copies and all
// MMAs; stages are double-buffered so the copies for chunk c + 1 overlap the
// MMAs of chunk c, across tile boundaries too (persistent CTAs), and the
// accumulators are double-buffered in TMEM so the epilogue of one tile
// overlaps the next.  Every wait is bounded and reports through *err.
//
// Shapes: X a multiple of 128, Z even, cin a multiple of 8, cout a multiple of
// 16 up to 64.  Tiles are 4 z-lines high for cout <= 32 (shared memory
// 2 x (75,776 + 864 cout) bytes), else 2 (2 x (50,176 + 864 cout)).  Other
// shapes use the gather kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "cnn_tc.cuh"
#include "xtg_cnn_internal.h"

namespace xtc {

namespace {

constexpr int TX = 128, TXS = TX + 2;  // output x-voxels per tile, staged with one halo each side
constexpr int TN_MAX = 64;

// per tile height TZ (output z-lines): 4 for cout <= 32, else 2 (shared memory)
template <int TZ>
struct TileDims {
  static constexpr int TZS = TZ + 2;                   // staged z-lines
  static constexpr int ROWS = 3 * TZS * TXS;           // staged voxels, one 32-byte row (16 channels) each
  static constexpr uint32_t BOX = ROWS * 32;           // bytes one TMA box writes
  static constexpr uint32_t A_STAGE = (BOX + 1023) / 1024 * 1024;  // stages stay aligned to the swizzle atom
};

// K-major operand with 32-byte rows in the 32-byte swizzle (16-byte chunk
// index XOR address bit 7, as TMA's SWIZZLE_32B writes it): the two 8-element
// K halves of a row are one 16-byte unit apart, 8-row groups 256 bytes apart.
// The swizzle is a function of the absolute shared-memory address, so a
// descriptor may start at any row.
__device__ __forceinline__ uint64_t sdesc_sw32(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)6 << 61);
}

__host__ __device__ constexpr uint32_t b_stage_bytes(int n) { return 27u * (uint32_t)n * 32u; }

// Persistent: each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// Warp 4 (one thread) issues the copies and MMAs of the CTA's whole chunk
// sequence through two shared-memory stages; the accumulators alternate
// between two TMEM buffers, so warps 0-3 (TMEM lanes 32w .. 32w + 31) drain
// tile i while tile i + 1 is computed.
template <int EPI, int TZ>
__global__ void __launch_bounds__(160, 1)
    k_conv_tile(const __grid_constant__ CUtensorMap tin, ConvShape s, const __nv_bfloat16 *__restrict__ wp,
                const float *__restrict__ bias, void *out, int *err) {
  using D = TileDims<TZ>;
  constexpr int TZS = D::TZS;
  constexpr uint32_t TA_STAGE = D::A_STAGE;
  extern __shared__ __align__(1024) uint8_t sm[];
  const int N = s.n;
  const uint32_t B_STAGE = b_stage_bytes(N);
  uint8_t *sA = sm, *sB = sm + 2 * TA_STAGE;
  __shared__ uint64_t full[2], empty[2], acc_full[2], acc_empty[2], done;
  __shared__ uint32_t tbase;
  __shared__ volatile int bad;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = (s.cin + 15) >> 4;
  const int XT = s.X / TX, ZT = s.Z / TZ;
  const int ntiles = XT * ZT * s.nb * s.Y;
  const int mine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const uint32_t acc_cols = tmem_cols(2 * TZ * N);
  const long long lim = 1ll << 24;
  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 4);
    }
    mbar_init(&done, 1);
    mbar_init_fence();
    bad = 0;
  }
  if (warp == 0) tmem_alloc(&tbase, acc_cols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (warp < 4) {  // both accumulator buffers start at zero
    for (int col = 0; col < 2 * TZ * N; col += 16) tmem_st16_zero(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  auto tile_of = [&](int tl, int &x0, int &z0, int &y, int &b) {
    int t = (int)blockIdx.x + tl * (int)gridDim.x;
    x0 = (t % XT) * TX;
    t /= XT;
    z0 = (t % ZT) * TZ;
    t /= ZT;
    y = t % s.Y;
    b = t / s.Y;
  };
  if (warp == 4) {
    if (lane == 0 && mine > 0) {
      const uint32_t idesc[3] = {idesc_bf16(N, 0, 0), idesc_bf16(2 * N, 0, 0), idesc_bf16(3 * N, 0, 0)};
      const int Q = mine * nchunk;
      int issued[2] = {0, 0}, landed[2] = {0, 0};
      auto load = [&](int q) {
        const int st = q & 1, c = q % nchunk;
        int x0, z0, y, b;
        tile_of(q / nchunk, x0, z0, y, b);
        uint8_t *a = sA + st * TA_STAGE;
        mbar_expect_tx(&full[st], D::BOX + B_STAGE);
        // channels 16c .. 16c + 15 (past cin: zero fill)
        tma_load_5d(a, &tin, 16 * c, x0 - 1, z0 - 1, y - 1, b, &full[st]);
        bulk_load(sB + st * B_STAGE, wp + (size_t)c * (B_STAGE / 2), B_STAGE, &full[st]);
        issued[st]++;
      };
      bool ok = true;
      load(0);
      if (Q > 1) load(1);
      for (int q = 0; q < Q && ok; q++) {
        const int st = q & 1, c = q % nchunk, tl = q / nchunk, ab = tl & 1;
        if (c == 0 && !mbar_wait(&acc_empty[ab], (uint32_t)(((tl >> 1) & 1) ^ 1), lim)) {
          ok = false;
          break;
        }
        if (!mbar_wait(&full[st], (uint32_t)(q >> 1) & 1u, lim)) {
          ok = false;
          break;
        }
        landed[st]++;
        tc_fence_after();
        // descriptors advance in 16-byte units: an A row by 2; a (dy, dx)
        // B block (2 halves x 3 dz x N rows x 16 bytes) by 6N, one dz block by N
        const uint32_t acc = tmem + (uint32_t)(ab * TZ * N);
        const uint64_t da0 = sdesc_sw32(smem_u32(sA + st * TA_STAGE) + (uint32_t)((TZS + 1) * TXS + 1) * 32);
        uint64_t db = sdesc(smem_u32(sB + st * B_STAGE), (uint32_t)N * 48, 128);
#pragma unroll
        for (int g = 0; g < 9; g++) {
          const int dy = g / 3 - 1, dx = g % 3 - 1;
#pragma unroll
          for (int zl = 0; zl < TZS; zl++) {
            // staged line zl (z = z0 - 1 + zl) feeds output lines zl - 2 .. zl
            // (relative to z0) through dz = +1, 0, -1; keep those inside the tile
            const int zf = zl - 2 < 0 ? 0 : zl - 2, zt = zl > TZ - 1 ? TZ - 1 : zl;
            const int cnt = zt - zf + 1, blk = zf - (zl - 2);
            mma_bf16(acc + (uint32_t)(zf * N), da0 + (uint64_t)(int64_t)(2 * ((dy * TZS + zl - 1) * TXS + dx)),
                     db + (uint64_t)(blk * N), idesc[cnt - 1], 1u);
          }
          db += (uint64_t)(6 * N);
        }
        mma_commit(&empty[st]);
        if (c == nchunk - 1) mma_commit(&acc_full[ab]);
        if (q >= 1 && q + 1 < Q) {
          // chunk q + 1 reuses the stage of chunk q - 1 once its MMAs are done
          if (!mbar_wait(&empty[(q - 1) & 1], (uint32_t)((q - 1) >> 1) & 1u, lim)) {
            ok = false;
            break;
          }
          load(q + 1);
        }
      }
      if (!ok || bad) {
        atomicExch(err, 1);
        bad = 1;
        // let the copies already issued land before the shared memory is released
        for (int st = 0; st < 2; st++)
          for (; landed[st] < issued[st]; landed[st]++) mbar_wait(&full[st], (uint32_t)landed[st] & 1u, lim);
      }
      mma_commit(&done);
      mbar_wait(&done, 0, lim);  // every MMA issued above has completed
    }
    __syncwarp();
  } else {
    // epilogue: warp w drains accumulator rows (x) 32w .. 32w + 31
    for (int tl = 0; tl < mine; tl++) {
      const int ab = tl & 1;
      if (!mbar_wait(&acc_full[ab], (uint32_t)(tl >> 1) & 1u, lim) || bad) {
        if (lane == 0) atomicExch(err, 1);
        bad = 1;
        break;
      }
      tc_fence_after();
      int x0, z0, y, b;
      tile_of(tl, x0, z0, y, b);
      for (int zo = 0; zo < TZ; zo++) {
        const size_t vox = (((size_t)b * s.Y + y) * s.X + x0 + warp * 32 + lane) * s.Z + z0 + zo;
        for (int n0 = 0; n0 < N; n0 += 16) {
          float v[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((ab * TZ + zo) * N + n0), v);
          if (EPI == 2) {
            float *o = reinterpret_cast<float *>(out) + vox * N + n0;
#pragma unroll
            for (int q = 0; q < 16; q += 4)
              *reinterpret_cast<float4 *>(o + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
          } else {
            __align__(16) __nv_bfloat16 h[16];
#pragma unroll
            for (int q = 0; q < 16; q++) {
              float t = v[q];
              if (EPI == 0) t = fmaxf(t + bias[n0 + q], 0.f);
              h[q] = __float2bfloat16_rn(t);
            }
            __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(out) + vox * N + n0;
            *reinterpret_cast<int4 *>(o) = *reinterpret_cast<const int4 *>(h);
            *reinterpret_cast<int4 *>(o + 8) = *reinterpret_cast<const int4 *>(h + 8);
          }
        }
      }
      // the buffer starts the CTA's next tile at zero
      for (int col = 0; col < TZ * N; col += 16)
        tmem_st16_zero(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ab * TZ * N + col));
      tmem_st_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[ab]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, acc_cols);
  }
}

// K-major W[n][kpad] (k = tap * cin + ci, tap = (dy+1)*9 + (dx+1)*3 + (dz+1))
// -> Wp[chunk][(ey+1)*3 + (ex+1)][half][dzi][n][8], ci = 16 chunk + 8 half + e,
// effective offsets (ey, ex, ez = 1 - dzi) = sign x (dy, dx, dz)
__global__ void k_pack_tile_w(int cin, int n, int kpad, int sign, const __nv_bfloat16 *__restrict__ w,
                              __nv_bfloat16 *__restrict__ wp) {
  const long long total = (long long)((cin + 15) / 16) * 27 * 2 * n * 8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int e = (int)(r % 8);
    r /= 8;
    const int nn = (int)(r % n);
    r /= n;
    const int dzi = (int)(r % 3);
    r /= 3;
    const int h = (int)(r % 2);
    r /= 2;
    const int g = (int)(r % 9);
    const int c = (int)(r / 9);
    const int ci = 16 * c + 8 * h + e;
    const int dy = sign * (g / 3 - 1), dx = sign * (g % 3 - 1), dz = sign * (1 - dzi);
    const int t = (dy + 1) * 9 + (dx + 1) * 3 + (dz + 1);
    wp[i] = ci < cin ? w[(size_t)nn * kpad + (size_t)t * cin + ci] : __float2bfloat16_rn(0.f);
  }
}

// ---------------------------------------------------------------------------
// Weight gradient on staged tiles (cout = 32, cin a multiple of 16, X a
// multiple of 128, Z even):
//   dW[dy, dx, dz][ci][co] = sum_v dY[v][co] X[v + (dy, dx, dz)][ci]
//                          = sum_u dY[u - (dy, 0, 0)][co] X[u + (0, dx, dz)][ci]
// (dY and X are zero outside the volume, so the substitution v = u - dy
// drops nothing).  In the second form one MMA covers the three dy taps along
// M and the three dz taps along N.  A CTA walks tiles u = 128 x-voxels x 2
// z-lines of one y-row y0 and keeps D[(dy, co)][(dx, dz, ci)] for up to three
// 16-channel input chunks in TMEM over all its tiles.  Per tile it stages, by
// TMA, one 32-byte row (16 channels) per voxel:
//   A (M x K, MN-major): dY rows y0 + 1, y0, y0 - 1 (dy = -1, 0, +1) x 2
//     channel halves = 6 boxes of 2 x 128 rows, stacked along M at a uniform
//     atom stride (M = 96; the MMA's rows 96..127 read the next box and are
//     discarded);
//   B (N x K, MN-major): per input chunk, the X halo of row y0
//     (130 x-voxels x 4 z-lines, zero fill outside); for (dx, output line z)
//     the three z-lines z - 1, z, z + 1 (dz = -1, 0, +1) are atoms one z-line
//     (130 rows) apart, and dx shifts the start row.
// K is the x-voxel: 16 rows per MMA.  Warp 4 (one thread) issues the copies
// and MMAs through two stages; warps 0-2 (TMEM lanes = (dy, co)) add the
// accumulators into dw once at the end.  Every wait is bounded.
constexpr int WG_TZ = 2;                                 // output z-lines per tile
constexpr uint32_t WG_XB = (WG_TZ + 2) * TXS * 32;       // one X box: 16,640 bytes
constexpr uint32_t WG_XS = (WG_XB + 1023) / 1024 * 1024; // its stride in a stage
constexpr uint32_t WG_DB = WG_TZ * TX * 32;              // one dY box: 8,192 bytes
constexpr uint32_t WG_A = 6 * WG_DB;                     // 3 y-rows x 2 channel halves
constexpr int WG_CPG = 3;                                // input chunks per CTA: 3 x 144 TMEM columns
constexpr uint32_t WG_SLACK = 16384;                     // past the second stage
constexpr int WG_N = 48;                                 // 3 dz x 16 channels

__host__ __device__ constexpr uint32_t wg_stage(int cpg) { return WG_A + (uint32_t)cpg * WG_XS; }

// MN-major operand, 32-byte swizzle: 16-element (32-byte) rows, one per K
// index, 8-row groups 256 bytes apart (SBO); MN atoms of 16 elements `lbo`
// bytes apart (LBO).
__device__ __forceinline__ uint64_t sdesc_mn_sw32(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(256 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

__global__ void __launch_bounds__(160, 1)
    k_wgrad_tile(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tdy, ConvShape s,
                 float *dw, int slices, int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t full[2], empty[2], acc_full;
  __shared__ uint32_t tbase;
  __shared__ volatile int bad;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = s.cin >> 4;
  const int cpg = nchunk < WG_CPG ? nchunk : WG_CPG;
  const uint32_t STAGE = wg_stage(cpg);
  const int grp = (int)blockIdx.x / slices, slice = (int)blockIdx.x % slices;
  const int c0 = grp * cpg, nck = nchunk - c0 < cpg ? nchunk - c0 : cpg;
  const int XT = s.X / TX, ZT = s.Z / WG_TZ;
  const int ntiles = XT * ZT * s.nb * s.Y;
  const int mine = ntiles > slice ? (ntiles - 1 - slice) / slices + 1 : 0;
  const long long lim = 1ll << 24;
  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&acc_full, 1);
    mbar_init_fence();
    bad = 0;
  }
  if (warp == 0) tmem_alloc(&tbase, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  const int ncols = nck * 3 * WG_N;
  if (warp < 4) {
    for (int col = 0; col < ncols; col += 16) tmem_st16_zero(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  auto tile_of = [&](int tl, int &x0, int &z0, int &y, int &b) {
    int t = slice + tl * slices;
    x0 = (t % XT) * TX;
    t /= XT;
    z0 = (t % ZT) * WG_TZ;
    t /= ZT;
    y = t % s.Y;
    b = t / s.Y;
  };
  if (warp == 4) {
    if (lane == 0) {
      bool ok = true;
      if (mine > 0) {
        const uint32_t idesc = idesc_bf16(WG_N, 1, 1);
        int issued[2] = {0, 0}, landed[2] = {0, 0};
        auto load = [&](int q) {
          const int st = q & 1;
          int x0, z0, y, b;
          tile_of(q, x0, z0, y, b);
          uint8_t *g = sm + st * STAGE;
          mbar_expect_tx(&full[st], 6 * WG_DB + (uint32_t)nck * WG_XB);
          // box j = dy + 1 holds dY row y0 - dy (zero fill outside)
          for (int j = 0; j < 3; j++)
            for (int h = 0; h < 2; h++) tma_load_5d(g + (j * 2 + h) * WG_DB, &tdy, 16 * h, x0, z0, y + 1 - j, b, &full[st]);
          for (int c = 0; c < nck; c++)
            tma_load_5d(g + WG_A + c * WG_XS, &tin, 16 * (c0 + c), x0 - 1, z0 - 1, y, b, &full[st]);
          issued[st]++;
        };
        load(0);
        if (mine > 1) load(1);
        for (int q = 0; q < mine && ok; q++) {
          const int st = q & 1;
          if (!mbar_wait(&full[st], (uint32_t)(q >> 1) & 1u, lim)) {
            ok = false;
            break;
          }
          landed[st]++;
          tc_fence_after();
          const uint32_t g = smem_u32(sm + st * STAGE);
          for (int c = 0; c < nck; c++) {
            for (int q3 = 0; q3 < 3; q3++) {  // dx = q3 - 1
              const uint32_t acc = tmem + (uint32_t)((c * 3 + q3) * WG_N);
#pragma unroll
              for (int zo = 0; zo < WG_TZ; zo++) {
#pragma unroll
                for (int ks = 0; ks < TX / 16; ks++) {
                  const uint64_t da = sdesc_mn_sw32(g + (uint32_t)(zo * TX + ks * 16) * 32, WG_DB);
                  const uint64_t db = sdesc_mn_sw32(g + WG_A + (uint32_t)c * WG_XS + (uint32_t)(zo * TXS + ks * 16 + q3) * 32,
                                                    TXS * 32);
                  mma_bf16(acc, da, db, idesc, 1u);
                }
              }
            }
          }
          mma_commit(&empty[st]);
          if (q >= 1 && q + 1 < mine) {
            // tile q + 1 reuses the stage of tile q - 1 once its MMAs are done
            if (!mbar_wait(&empty[(q - 1) & 1], (uint32_t)((q - 1) >> 1) & 1u, lim)) {
              ok = false;
              break;
            }
            load(q + 1);
          }
        }
        if (!ok) {
          // let the copies already issued land before the shared memory is released
          for (int st = 0; st < 2; st++)
            for (; landed[st] < issued[st]; landed[st]++) mbar_wait(&full[st], (uint32_t)landed[st] & 1u, lim);
        }
      }
      if (!ok) {
        atomicExch(err, 1);
        bad = 1;
      }
      mma_commit(&acc_full);  // arrives once every MMA issued above has completed
    }
    __syncwarp();
  } else {
    const bool ready = mbar_wait(&acc_full, 0, lim);
    if (!ready) {
      if (lane == 0) atomicExch(err, 1);
      bad = 1;
    }
    tc_fence_after();
    if (warp < 3 && ready && !bad && mine > 0) {
      // TMEM lane 32 w + co holds dy = w - 1, output channel co
      for (int c = 0; c < nck; c++)
        for (int q3 = 0; q3 < 3; q3++)
          for (int n0 = 0; n0 < WG_N; n0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((c * 3 + q3) * WG_N + n0), v);
            const int tap = warp * 9 + q3 * 3 + n0 / 16;
            float *o = dw + ((size_t)tap * s.cin + (size_t)(c0 + c) * 16) * 32 + lane;
#pragma unroll
            for (int i = 0; i < 16; i++) atomicAdd(o + (size_t)i * 32, v[i]);
          }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, 512);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

// tile height for a shape: 4 z-lines when cout <= 32 and Z allows, else 2
static int tile_tz(const ConvShape &s) { return (s.n <= 32 && s.Z % 4 == 0) ? 4 : 2; }

bool wgrad_tile_supported(const ConvShape &s) {
  return s.nb >= 1 && s.Y >= 1 && s.X >= TX && s.X % TX == 0 && s.Z >= WG_TZ && s.Z % WG_TZ == 0 && s.cin >= 16 &&
         s.cin % 16 == 0 && s.n == 32 && (long long)(s.X / TX) * (s.Z / WG_TZ) * s.nb * s.Y < (1ll << 31) &&
         encode_fn() != nullptr;
}

// activations [nb][Y][X][Z][c] seen as (c, x, z, y, b), boxes of 16 channels
static bool encode_act(CUtensorMap *m, const __nv_bfloat16 *p, const ConvShape &s, int c, int bx, int bz) {
  const cuuint64_t C2 = (cuuint64_t)c * 2;
  const cuuint64_t dims[5] = {(cuuint64_t)c, (cuuint64_t)s.X, (cuuint64_t)s.Z, (cuuint64_t)s.Y, (cuuint64_t)s.nb};
  const cuuint64_t strides[4] = {(cuuint64_t)s.Z * C2, C2, (cuuint64_t)s.X * s.Z * C2, (cuuint64_t)s.Y * s.X * s.Z * C2};
  const cuuint32_t box[5] = {16, (cuuint32_t)bx, (cuuint32_t)bz, 1, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16 *>(p), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t conv_wgrad_tile(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, float *dw,
                            int *err, cudaStream_t st) {
  if (!wgrad_tile_supported(s)) return cudaErrorNotSupported;
  CUtensorMap mi, md;
  if (!encode_act(&mi, in, s, s.cin, TXS, WG_TZ + 2) || !encode_act(&md, dout, s, s.n, TX, WG_TZ))
    return cudaErrorNotSupported;
  const int nchunk = s.cin / 16, cpg = std::min(nchunk, WG_CPG);
  const int groups = (nchunk + cpg - 1) / cpg;
  static int sms = 0;
  cudaError_t e;
  if (!sms) {
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  }
  const long long ntiles = (long long)(s.X / TX) * (s.Z / WG_TZ) * s.nb * s.Y;
  const int slices = (int)std::max(1ll, std::min(ntiles, (long long)std::max(1, sms / groups)));
  const size_t smem = 2 * (size_t)wg_stage(cpg) + WG_SLACK;
  e = cudaFuncSetAttribute((const void *)k_wgrad_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_wgrad_tile<<<(unsigned)(groups * slices), 160, smem, st>>>(mi, md, s, dw, slices, err);
  return cudaGetLastError();
}

bool conv_tile_supported(const ConvShape &s) {
  return s.nb >= 1 && s.Y >= 1 && s.X >= TX && s.X % TX == 0 && s.Z >= 2 && s.Z % 2 == 0 && s.cin >= 8 &&
         s.cin % 8 == 0 && s.n >= 16 && s.n % 16 == 0 && s.n <= TN_MAX &&
         (long long)(s.X / TX) * (s.Z / 2) * s.nb * s.Y < (1ll << 31) && encode_fn() != nullptr;
}

size_t conv_tile_wp_elems(int cin, int n) { return (size_t)((cin + 15) / 16) * 27 * 2 * n * 8; }

cudaError_t conv_tile_pack(int cin, int n, int kpad, int sign, const __nv_bfloat16 *w, __nv_bfloat16 *wp,
                           cudaStream_t st) {
  const long long total = (long long)conv_tile_wp_elems(cin, n);
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 4096);
  k_pack_tile_w<<<grid, 256, 0, st>>>(cin, n, kpad, sign, w, wp);
  return cudaGetLastError();
}

cudaError_t conv_forward_tile(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *wp, const float *bias,
                              void *out, int epi, int sign, int *err, cudaStream_t st) {
  if (!conv_tile_supported(s) || (epi == 0 && !bias) || epi < 0 || epi > 2 || (sign != 1 && sign != -1))
    return cudaErrorNotSupported;
  // activations [nb][Y][X][Z][cin] seen as (c, x, z, y, b): the box lands x-fastest
  CUtensorMap m;
  const cuuint64_t C2 = (cuuint64_t)s.cin * 2;
  const cuuint64_t dims[5] = {(cuuint64_t)s.cin, (cuuint64_t)s.X, (cuuint64_t)s.Z, (cuuint64_t)s.Y,
                              (cuuint64_t)s.nb};
  const cuuint64_t strides[4] = {(cuuint64_t)s.Z * C2, C2, (cuuint64_t)s.X * s.Z * C2,
                                 (cuuint64_t)s.Y * s.X * s.Z * C2};
  const int tz = tile_tz(s);
  const cuuint32_t box[5] = {16, TXS, (cuuint32_t)tz + 2, 3, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  if (encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16 *>(in), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorNotSupported;
  typedef void (*K)(const CUtensorMap, ConvShape, const __nv_bfloat16 *, const float *, void *, int *);
  K k;
  // the sign lives in the packed weights
  if (tz == 4)
    k = epi == 0 ? k_conv_tile<0, 4> : epi == 1 ? k_conv_tile<1, 4> : k_conv_tile<2, 4>;
  else
    k = epi == 0 ? k_conv_tile<0, 2> : epi == 1 ? k_conv_tile<1, 2> : k_conv_tile<2, 2>;
  const size_t smem =
      2 * ((size_t)(tz == 4 ? TileDims<4>::A_STAGE : TileDims<2>::A_STAGE) + b_stage_bytes(s.n));
  cudaError_t e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  }
  const long long ntiles = (long long)(s.X / TX) * (s.Z / tz) * s.nb * s.Y;
  const unsigned grid = (unsigned)std::min<long long>(ntiles, sms);  // one CTA per SM (shared memory)
  k<<<grid, 160, smem, st>>>(m, s, wp, bias, out, err);
  return cudaGetLastError();
}

}  // namespace xtc
