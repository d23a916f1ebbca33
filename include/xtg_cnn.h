/*
 * xtg_cnn.h -- C ABI of the learned warm start for the B200 TIMBIR engine:
 * BF16 3D convolutions on the tcgen05 tensor cores and the small 3D
 * encoder-decoder network built from them.
 *
 * No reference counterpart: gromitsun/timbir-python has no learned warm
 * start; the reference starts ICD from zero or a coarser stage
 * (initObject, Source_Code_4D_Fast/XT_ICD_update.c:443-536).
 *
 * Volumes are channels-last BF16 device buffers [nb][Y][X][Z][C] (C a
 * multiple of 8).  All functions return 0 or a negative status
 * (XTG_E_* of xtg.h); xtg_last_error() describes the failure.
 */
#ifndef XTG_CNN_H
#define XTG_CNN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 3x3x3 convolution, padding 1, on device buffers (the caller's stream 0).
 * w: K-major weights [cout][kpad], k = tap*cin + ci, tap = (dy+1)*9 +
 * (dx+1)*3 + (dz+1), kpad = 27*cin rounded up to 64 (zero tail).
 * epi 0: out = ReLU(acc + bias) in BF16; 1: out = acc in BF16; 2: out = acc
 * in FP32.  sign +1 gathers in[v + d], -1 gathers in[v - d] (the input
 * gradient, with w holding the transposed weights [cin][27*cout]). */
int xtc_conv3d(const void *in, const void *w, const float *bias, void *out, int32_t nb, int32_t Y, int32_t X,
               int32_t Z, int32_t cin, int32_t cout, int32_t kpad, int32_t epi, int32_t sign);

/* Weight gradient: dw[(tap*cin + ci)][cout] += sum_v in[v + d(tap)][ci] dout[v][cout] (FP32 atomics). */
int xtc_conv3d_wgrad(const void *in, const void *dout, float *dw, int32_t nb, int32_t Y, int32_t X, int32_t Z,
                     int32_t cin, int32_t cout);

#ifdef __cplusplus
}
#endif
#endif
