// xtg_cnn_internal.h -- shared declarations of the warm-start network's kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace xtc {

// channels-last volume [nb][Y][X][Z][cin] convolved to n output channels
struct ConvShape {
  int nb, Y, X, Z;
  int cin;   // input channels as stored (multiple of 8)
  int n;     // output channels (multiple of 16, <= 256)
  int kpad;  // K-major weight row length: 27 * cin rounded up to 64
};

cudaError_t conv_forward(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                         void *out, int epi, int sign, int *err, cudaStream_t st);
// the first layer (2 FP32 input channels, the input packing fused in): w64 [n][64], k = 2 tap + channel
cudaError_t conv_first_pack(int n, int cin, int kpad, const __nv_bfloat16 *w, __nv_bfloat16 *w64, cudaStream_t st);
cudaError_t conv_first(int nb, int Y, int X, int Z, const float *a, const float *b, float scale,
                       const __nv_bfloat16 *w64, const float *bias, int n, __nv_bfloat16 *out, int *err,
                       cudaStream_t st);
// the TMA-staged tile kernel (cnn_conv_tile.cu): X a multiple of 128, Z even,
// n <= 64; weights pre-packed by conv_tile_pack into conv_tile_wp_elems values
bool conv_tile_supported(const ConvShape &s);
size_t conv_tile_wp_elems(int cin, int n);
cudaError_t conv_tile_pack(int cin, int n, int kpad, int sign, const __nv_bfloat16 *w, __nv_bfloat16 *wp,
                           cudaStream_t st);
cudaError_t conv_forward_tile(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *wp, const float *bias,
                              void *out, int epi, int sign, int *err, cudaStream_t st);
// weight gradient: the TMA tile kernel where wgrad_tile_supported (cout 32,
// cin a multiple of 16, X a multiple of 128, Z even), else the gather kernel;
// path 1 forces the gather kernel, 2 the tile kernel (cudaErrorNotSupported
// where it does not apply)
cudaError_t conv_wgrad(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, float *dw, int *err,
                       cudaStream_t st, int path = 0);
bool wgrad_tile_supported(const ConvShape &s);
cudaError_t conv_wgrad_tile(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, float *dw,
                            int *err, cudaStream_t st);

void pack_input(long long nv, const float *a, const float *b, float scale, __nv_bfloat16 *out, cudaStream_t st);
void avgpool(int nb, int Y, int X, int Z, int C, const __nv_bfloat16 *in, __nv_bfloat16 *out, cudaStream_t st);
void avgpool_back(int nb, int Y, int X, int Z, int C, const float *dout, float *din, cudaStream_t st);
void up_concat(int nb, int Y, int X, int Z, int Ca, int Cb, const __nv_bfloat16 *a, const __nv_bfloat16 *skip,
               __nv_bfloat16 *out, cudaStream_t st);
void up_concat_back(int nb, int Y, int X, int Z, int Ca, int Cb, const float *dout, float *da, float *dskip,
                    cudaStream_t st);
void relu_back(long long nv, int C, const float *dpost, const __nv_bfloat16 *post, __nv_bfloat16 *dpre, float *dbias,
               cudaStream_t st);
void to_f32(long long n, const __nv_bfloat16 *a, float *b, cudaStream_t st);
void head(long long nv, int C, const __nv_bfloat16 *h, const float *w, const float *bias, const float *base, float scale,
          float *y, const float *target, double *loss, float *dh32, float *dw, float *db, cudaStream_t st);
void pack_weights(int cin_real, int cin, int cout, int kpad, int kpad_t, const float *P, __nv_bfloat16 *W,
                  __nv_bfloat16 *Wt, cudaStream_t st);
void fold_wgrad(int cin_real, int cin, int cout, const float *g, float *out, cudaStream_t st);
void adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
          cudaStream_t st);
void crop(int np, const float *const *src, const int4 *org, int Y, int X, int Z, int py, int px, int pz, float *dst,
          cudaStream_t st);

cudaError_t wait_selftest(int arrive, long long limit, int *err, cudaStream_t st);
}  // namespace xtc
