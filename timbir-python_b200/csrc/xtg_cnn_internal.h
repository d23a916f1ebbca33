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
cudaError_t conv_wgrad(const ConvShape &s, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, float *dw, int *err,
                       cudaStream_t st);

}  // namespace xtc
