// cnn_ops.cu -- the warm-start network's non-convolution kernels: input
// packing, 2x average pooling, nearest 2x upsampling with skip concatenation,
// ReLU and bias gradients, the 1x1 output head with the loss, weight packing
// and the Adam update.  Channels-last BF16 volumes [nb][Y][X][Z][C].
#include <cuda_bf16.h>

#include "xtg_cnn_internal.h"

namespace xtc {

static unsigned blocks(long long n, int t = 256) {
  long long b = (n + t - 1) / t;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}
#define GRID_STRIDE(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// two FP32 volumes [nb][Y][X][Z] -> BF16 [..][8] (channels 0, 1; rest 0), times scale
__global__ void k_pack_input(long long nv, const float *a, const float *b, float scale, __nv_bfloat16 *out) {
  GRID_STRIDE(v, nv) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int c = 0; c < 8; c++) h[c] = __float2bfloat16_rn(0.f);
    h[0] = __float2bfloat16_rn(a[v] * scale);
    h[1] = __float2bfloat16_rn(b[v] * scale);
    *reinterpret_cast<int4 *>(out + v * 8) = *reinterpret_cast<const int4 *>(h);
  }
}

// 2x2x2 average pooling (dims even)
__global__ void k_avgpool(int nb, int Y, int X, int Z, int C, const __nv_bfloat16 *in, __nv_bfloat16 *out) {
  const int Yo = Y / 2, Xo = X / 2, Zo = Z / 2;
  const long long n = (long long)nb * Yo * Xo * Zo * C;
  GRID_STRIDE(i, n) {
    long long r = i;
    const int c = (int)(r % C);
    r /= C;
    const int z = (int)(r % Zo);
    r /= Zo;
    const int x = (int)(r % Xo);
    r /= Xo;
    const int y = (int)(r % Yo);
    const int b = (int)(r / Yo);
    float s = 0.f;
    for (int d = 0; d < 8; d++) {
      const int yy = 2 * y + (d >> 2), xx = 2 * x + ((d >> 1) & 1), zz = 2 * z + (d & 1);
      s += __bfloat162float(in[((((size_t)b * Y + yy) * X + xx) * Z + zz) * C + c]);
    }
    out[i] = __float2bfloat16_rn(s * 0.125f);
  }
}

// the same pooling on 8-channel groups (C a multiple of 8): 16-byte loads and
// stores, each channel summed in the same order as above
__global__ void k_avgpool8(int nb, int Y, int X, int Z, int G, const int4 *in, int4 *out) {
  const int Yo = Y / 2, Xo = X / 2, Zo = Z / 2;
  const long long n = (long long)nb * Yo * Xo * Zo * G;
  GRID_STRIDE(i, n) {
    long long r = i;
    const int g = (int)(r % G);
    r /= G;
    const int z = (int)(r % Zo);
    r /= Zo;
    const int x = (int)(r % Xo);
    r /= Xo;
    const int y = (int)(r % Yo);
    const int b = (int)(r / Yo);
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int d = 0; d < 8; d++) {
      const int yy = 2 * y + (d >> 2), xx = 2 * x + ((d >> 1) & 1), zz = 2 * z + (d & 1);
      const int4 q = __ldg(in + ((((size_t)b * Y + yy) * X + xx) * Z + zz) * G + g);
      const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&q);
#pragma unroll
      for (int c = 0; c < 8; c++) s[c] += __bfloat162float(h[c]);
    }
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int c = 0; c < 8; c++) o[c] = __float2bfloat16_rn(s[c] * 0.125f);
    out[i] = *reinterpret_cast<const int4 *>(o);
  }
}

// gradient of the pooling, added into dIn (FP32 accumulation buffer)
__global__ void k_avgpool_back(int nb, int Y, int X, int Z, int C, const float *dout, float *din) {
  const long long n = (long long)nb * Y * X * Z * C;
  GRID_STRIDE(i, n) {
    long long r = i;
    const int c = (int)(r % C);
    r /= C;
    const int z = (int)(r % Z);
    r /= Z;
    const int x = (int)(r % X);
    r /= X;
    const int y = (int)(r % Y);
    const int b = (int)(r / Y);
    din[i] += 0.125f * dout[((((size_t)b * (Y / 2) + y / 2) * (X / 2) + x / 2) * (Z / 2) + z / 2) * C + c];
  }
}

// out[v] = [up2(a)[v] (Ca channels), skip[v] (Cb channels)] at the fine grid
__global__ void k_up_concat(int nb, int Y, int X, int Z, int Ca, int Cb, const __nv_bfloat16 *a,
                            const __nv_bfloat16 *skip, __nv_bfloat16 *out) {
  const int C = Ca + Cb;
  const long long n = (long long)nb * Y * X * Z * C;
  GRID_STRIDE(i, n) {
    long long r = i;
    const int c = (int)(r % C);
    r /= C;
    const int z = (int)(r % Z);
    r /= Z;
    const int x = (int)(r % X);
    r /= X;
    const int y = (int)(r % Y);
    const int b = (int)(r / Y);
    out[i] = c < Ca ? a[((((size_t)b * (Y / 2) + y / 2) * (X / 2) + x / 2) * (Z / 2) + z / 2) * Ca + c]
                    : skip[((((size_t)b * Y + y) * X + x) * Z + z) * Cb + (c - Ca)];
  }
}

// the same on 8-channel groups (Ca, Cb multiples of 8): one 16-byte copy per
// group, consecutive threads on consecutive output groups; GA, GB fixed at
// compile time (0: taken from the arguments) and 32-bit indices (n < 2^31)
template <int GA, int GB>
__global__ void k_up_concat8(int nb, int Y, int X, int Z, int ga, int gb, const int4 *__restrict__ a,
                             const int4 *__restrict__ skip, int4 *__restrict__ out) {
  const unsigned Ga = GA ? GA : ga, Gb = GB ? GB : gb, G = Ga + Gb;
  const unsigned n = (unsigned)nb * Y * X * Z * G;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned v = i / G, g = i - v * G;
    if (g < Ga) {
      const unsigned z = v % Z, r1 = v / Z, x = r1 % X, r2 = r1 / X;  // r2 = b * Y + y
      const unsigned cv = ((r2 >> 1) * (X >> 1) + (x >> 1)) * (Z >> 1) + (z >> 1);  // Y even: b*Y/2 + y/2
      out[i] = __ldg(a + (size_t)cv * Ga + g);
    } else {
      out[i] = __ldg(skip + (size_t)v * Gb + (g - Ga));
    }
  }
}

// gradient of k_up_concat: da (coarse, FP32, overwritten) and dskip (added into FP32)
__global__ void k_up_concat_back(int nb, int Y, int X, int Z, int Ca, int Cb, const float *dout, float *da,
                                 float *dskip) {
  const int C = Ca + Cb;
  const int Yo = Y / 2, Xo = X / 2, Zo = Z / 2;
  const long long na = (long long)nb * Yo * Xo * Zo * Ca;
  GRID_STRIDE(i, na) {
    long long r = i;
    const int c = (int)(r % Ca);
    r /= Ca;
    const int z = (int)(r % Zo);
    r /= Zo;
    const int x = (int)(r % Xo);
    r /= Xo;
    const int y = (int)(r % Yo);
    const int b = (int)(r / Yo);
    float s = 0.f;
    for (int d = 0; d < 8; d++) {
      const int yy = 2 * y + (d >> 2), xx = 2 * x + ((d >> 1) & 1), zz = 2 * z + (d & 1);
      s += dout[((((size_t)b * Y + yy) * X + xx) * Z + zz) * C + c];
    }
    da[i] = s;
  }
  const long long nskip = (long long)nb * Y * X * Z * Cb;
  GRID_STRIDE(i, nskip) {
    const long long v = i / Cb;
    const int c = (int)(i - v * Cb);
    dskip[i] += dout[v * C + Ca + c];
  }
}

// dpre = dpost * (post > 0), FP32 in -> BF16 out; the bias gradient summed per channel
__global__ void k_relu_back(long long nv, int C, const float *dpost, const __nv_bfloat16 *post, __nv_bfloat16 *dpre,
                            float *dbias) {
  extern __shared__ float sb[];
  for (int c = threadIdx.x; c < C; c += blockDim.x) sb[c] = 0.f;
  __syncthreads();
  const long long n = nv * C;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % C);
    const float g = __bfloat162float(post[i]) > 0.f ? dpost[i] : 0.f;
    dpre[i] = __float2bfloat16_rn(g);
    if (g != 0.f) atomicAdd(&sb[c], g);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&dbias[c], sb[c]);
}

// BF16 -> FP32 conversion (input gradients of the convolutions are produced in FP32 directly)
__global__ void k_to_f32(long long n, const __nv_bfloat16 *a, float *b) {
  GRID_STRIDE(i, n) b[i] = __bfloat162float(a[i]);
}

// 1x1 head: y[v] = base[v] + (sum_c h[v][c] w[c] + bias) / scale; optional loss
// against target and its gradient w.r.t. h (BF16), w (FP32 atomics), bias.
// loss = mean((y - target)^2 * scale^2), accumulated in FP64.
__global__ void k_head(long long nv, int C, const __nv_bfloat16 *h, const float *w, const float *bias,
                       const float *base, float scale, float *y, const float *target, double *loss, float *dh32,
                       float *dw, float *db, float inv_n) {
  extern __shared__ float sh[];  // [C] dw partials, [1] db partial
  for (int c = threadIdx.x; c <= C; c += blockDim.x) sh[c] = 0.f;
  __syncthreads();
  double lsum = 0.0;
  GRID_STRIDE(v, nv) {
    float acc = bias[0];
    if (C % 8 == 0) {
      for (int c0 = 0; c0 < C; c0 += 8) {
        const int4 q = __ldg(reinterpret_cast<const int4 *>(h + v * C + c0));
        const __nv_bfloat16 *hq = reinterpret_cast<const __nv_bfloat16 *>(&q);
#pragma unroll
        for (int c = 0; c < 8; c++) acc += __bfloat162float(hq[c]) * w[c0 + c];
      }
    } else {
      for (int c = 0; c < C; c++) acc += __bfloat162float(h[v * C + c]) * w[c];
    }
    const float out = base[v] + acc / scale;
    if (y) y[v] = out;
    if (target) {
      const float diff = (out - target[v]) * scale;
      lsum += (double)diff * diff;
      const float g = 2.f * diff * inv_n;  // d loss / d acc
      for (int c = 0; c < C; c++) {
        dh32[v * C + c] = g * w[c];
        atomicAdd(&sh[c], g * __bfloat162float(h[v * C + c]));
      }
      atomicAdd(&sh[C], g);
    }
  }
  if (target) {
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum * inv_n);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&dw[c], sh[c]);
    if (threadIdx.x == 0) atomicAdd(db, sh[C]);
  }
}

// master weights P[(tap*cin + ci)][cout] (FP32) -> W[cout][kpad] and Wt[ci][kpad_t] (BF16)
__global__ void k_pack_weights(int cin_real, int cin, int cout, int kpad, int kpad_t, const float *P,
                               __nv_bfloat16 *W, __nv_bfloat16 *Wt) {
  const long long n = (long long)cout * kpad;
  GRID_STRIDE(i, n) {
    const int co = (int)(i / kpad), k = (int)(i % kpad);
    float v = 0.f;
    if (k < 27 * cin) {
      const int tap = k / cin, ci = k % cin;
      if (ci < cin_real) v = P[((size_t)tap * cin_real + ci) * cout + co];
    }
    W[i] = __float2bfloat16_rn(v);
  }
  if (!Wt) return;
  const long long nt = (long long)cin * kpad_t;
  GRID_STRIDE(i, nt) {
    const int ci = (int)(i / kpad_t), k = (int)(i % kpad_t);
    float v = 0.f;
    if (k < 27 * cout && ci < cin_real) {
      const int tap = k / cout, co = k % cout;
      v = P[((size_t)tap * cin_real + ci) * cout + co];
    }
    Wt[i] = __float2bfloat16_rn(v);
  }
}

// the weight gradient rows of a padded input layer ([(tap*cin + ci)][cout],
// cin padded) folded to the master layout ([(tap*cin_real + ci)][cout])
__global__ void k_fold_wgrad(int cin_real, int cin, int cout, const float *g, float *out) {
  const long long n = 27LL * cin_real * cout;
  GRID_STRIDE(i, n) {
    const int co = (int)(i % cout);
    const long long r = i / cout;
    const int tap = (int)(r / cin_real), ci = (int)(r % cin_real);
    out[i] = g[((size_t)tap * cin + ci) * cout + co];
  }
}

// Adam (Kingma & Ba 2015) with bias correction
__global__ void k_adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  GRID_STRIDE(i, n) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// patch batch: dst[p] = src_vol[p][y0:y0+py][x0:x0+px][z0:z0+pz]
__global__ void k_crop(int np, const float *const *src, const int4 *org, int Y, int X, int Z, int py, int px, int pz,
                       float *dst) {
  const long long n = (long long)np * py * px * pz;
  GRID_STRIDE(i, n) {
    long long r = i;
    const int z = (int)(r % pz);
    r /= pz;
    const int x = (int)(r % px);
    r /= px;
    const int y = (int)(r % py);
    const int p = (int)(r / py);
    const int4 o = org[p];
    dst[i] = src[o.w][(((size_t)(o.x + y)) * X + (o.y + x)) * Z + (o.z + z)];
  }
}

// ---------------------------------------------------------------- launchers
void crop(int np, const float *const *src, const int4 *org, int Y, int X, int Z, int py, int px, int pz, float *dst,
          cudaStream_t st) {
  k_crop<<<blocks((long long)np * py * px * pz), 256, 0, st>>>(np, src, org, Y, X, Z, py, px, pz, dst);
}
void pack_input(long long nv, const float *a, const float *b, float scale, __nv_bfloat16 *out, cudaStream_t st) {
  k_pack_input<<<blocks(nv), 256, 0, st>>>(nv, a, b, scale, out);
}
void avgpool(int nb, int Y, int X, int Z, int C, const __nv_bfloat16 *in, __nv_bfloat16 *out, cudaStream_t st) {
  if (C % 8 == 0)
    k_avgpool8<<<blocks((long long)nb * Y * X * Z * C / 64), 256, 0, st>>>(
        nb, Y, X, Z, C / 8, reinterpret_cast<const int4 *>(in), reinterpret_cast<int4 *>(out));
  else
    k_avgpool<<<blocks((long long)nb * Y * X * Z * C / 8), 256, 0, st>>>(nb, Y, X, Z, C, in, out);
}
void avgpool_back(int nb, int Y, int X, int Z, int C, const float *dout, float *din, cudaStream_t st) {
  k_avgpool_back<<<blocks((long long)nb * Y * X * Z * C), 256, 0, st>>>(nb, Y, X, Z, C, dout, din);
}
void up_concat(int nb, int Y, int X, int Z, int Ca, int Cb, const __nv_bfloat16 *a, const __nv_bfloat16 *skip,
               __nv_bfloat16 *out, cudaStream_t st) {
  const long long n8 = (long long)nb * Y * X * Z * (Ca + Cb) / 8;
  if (Ca % 8 == 0 && Cb % 8 == 0 && Y % 2 == 0 && n8 < (1ll << 31)) {
    const int ga = Ca / 8, gb = Cb / 8;
    auto k = (ga == 6 && gb == 4)   ? k_up_concat8<6, 4>
             : (ga == 8 && gb == 6)  ? k_up_concat8<8, 6>
             : (ga == 12 && gb == 8) ? k_up_concat8<12, 8>
                                     : k_up_concat8<0, 0>;
    k<<<blocks(n8), 256, 0, st>>>(nb, Y, X, Z, ga, gb, reinterpret_cast<const int4 *>(a),
                                  reinterpret_cast<const int4 *>(skip), reinterpret_cast<int4 *>(out));
  } else
    k_up_concat<<<blocks((long long)nb * Y * X * Z * (Ca + Cb)), 256, 0, st>>>(nb, Y, X, Z, Ca, Cb, a, skip, out);
}
void up_concat_back(int nb, int Y, int X, int Z, int Ca, int Cb, const float *dout, float *da, float *dskip,
                    cudaStream_t st) {
  k_up_concat_back<<<blocks((long long)nb * Y * X * Z * Cb), 256, 0, st>>>(nb, Y, X, Z, Ca, Cb, dout, da, dskip);
}
void relu_back(long long nv, int C, const float *dpost, const __nv_bfloat16 *post, __nv_bfloat16 *dpre, float *dbias,
               cudaStream_t st) {
  k_relu_back<<<blocks(nv * C), 256, C * sizeof(float), st>>>(nv, C, dpost, post, dpre, dbias);
}
void to_f32(long long n, const __nv_bfloat16 *a, float *b, cudaStream_t st) {
  k_to_f32<<<blocks(n), 256, 0, st>>>(n, a, b);
}
void head(long long nv, int C, const __nv_bfloat16 *h, const float *w, const float *bias, const float *base, float scale,
          float *y, const float *target, double *loss, float *dh32, float *dw, float *db, cudaStream_t st) {
  k_head<<<blocks(nv), 256, (C + 1) * sizeof(float), st>>>(nv, C, h, w, bias, base, scale, y, target, loss, dh32, dw,
                                                            db, 1.f / (float)nv);
}
void pack_weights(int cin_real, int cin, int cout, int kpad, int kpad_t, const float *P, __nv_bfloat16 *W,
                  __nv_bfloat16 *Wt, cudaStream_t st) {
  k_pack_weights<<<blocks((long long)cout * kpad), 256, 0, st>>>(cin_real, cin, cout, kpad, kpad_t, P, W, Wt);
}
void fold_wgrad(int cin_real, int cin, int cout, const float *g, float *out, cudaStream_t st) {
  k_fold_wgrad<<<blocks(27LL * cin_real * cout), 256, 0, st>>>(cin_real, cin, cout, g, out);
}
void adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
          cudaStream_t st) {
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  k_adam<<<blocks(n), 256, 0, st>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
}

}  // namespace xtc
