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

/* xtc_conv3d with the kernel chosen: XTC_CONV_AUTO (what xtc_conv3d does), XTC_CONV_GATHER (operands
 * gathered per K stage by the CTA's threads) or XTC_CONV_TILE (input tile staged once by TMA, every tap
 * a shifted view of it; X a multiple of 128, Z even, cout <= 64, else XTG_E_ARG).  The tile kernel is
 * used by AUTO wherever it applies.  Its packed weights go to one buffer the library keeps: calls from
 * several host threads must be serialised. */
enum { XTC_CONV_AUTO = 0, XTC_CONV_GATHER = 1, XTC_CONV_TILE = 2 };
int xtc_conv3d_path(const void *in, const void *w, const float *bias, void *out, int32_t nb, int32_t Y, int32_t X,
                    int32_t Z, int32_t cin, int32_t cout, int32_t kpad, int32_t epi, int32_t sign, int32_t path);

/* Weight gradient: dw[(tap*cin + ci)][cout] += sum_v in[v + d(tap)][ci] dout[v][cout] (FP32 atomics). */
int xtc_conv3d_wgrad(const void *in, const void *dout, float *dw, int32_t nb, int32_t Y, int32_t X, int32_t Z,
                     int32_t cin, int32_t cout);

/* xtc_conv3d_wgrad with the kernel chosen: XTC_CONV_AUTO (what xtc_conv3d_wgrad does), XTC_CONV_GATHER
 * (operands gathered and transposed per K stage by the CTA's threads) or XTC_CONV_TILE (dout and the input
 * halo staged by TMA per tile of 128 x 2 voxels, the three dy taps stacked along M and the three dz taps
 * along N of each MMA; cout 32, cin a multiple of 16, X a multiple of 128, Z even, else XTG_E_ARG).  AUTO
 * uses the tile kernel wherever it applies. */
int xtc_conv3d_wgrad_path(const void *in, const void *dout, float *dw, int32_t nb, int32_t Y, int32_t X, int32_t Z,
                          int32_t cin, int32_t cout, int32_t path);

/* ---- the warm-start network ------------------------------------------------
 * A 3D encoder-decoder over channels-last volumes: four levels with 32, 48,
 * 64 and 96 channels, two 3x3x3 convolutions + ReLU per level on each side,
 * 2x average pooling down, nearest 2x upsampling + skip concatenation up and
 * a 1x1 head.  Input: the FBP image and a start image (FP32 [nb][Y][X][Z]
 * each, the engine's device layout with nb = frames); output: start image +
 * correction (the `icd` argument below is the start image).  Y, X, Z must be multiples of 8.  About 1.44 M
 * FP32 master parameters; BF16 weights and activations, FP32 accumulation. */
/* Health check of the bounded waits the tensor-core kernels use on their
 * mbarriers: one CTA waits `polls` polls on a barrier that it has arrived on
 * (arrive != 0: returns 0) or that nothing will complete (arrive == 0: the
 * wait gives up, sets the device error flag, and the call returns
 * XTG_E_TIMEOUT; nothing is in flight, the context stays usable).  No
 * reference counterpart. */
int xtc_wait_selftest(int32_t arrive, int64_t polls);

typedef struct xtc_net xtc_net;

/* He-initialised weights from the seed; the head starts at zero, so the new
 * network returns its ICD input unchanged. */
int xtc_net_create(uint64_t seed, xtc_net **net);
void xtc_net_destroy(xtc_net *net);
int64_t xtc_net_param_count(const xtc_net *net);
/* which = 0: parameters, 1: gradients of the last xtc_net_backward (host copy) */
int xtc_net_get_params(const xtc_net *net, float *host, int32_t which);
int xtc_net_set_params(xtc_net *net, const float *host);
int xtc_net_save(const xtc_net *net, const char *path);
int xtc_net_load(xtc_net *net, const char *path);
/* out = network(fbp, icd) on device buffers */
int xtc_net_forward(xtc_net *net, const float *fbp, const float *icd, float *out, int32_t nb, int32_t Y, int32_t X,
                    int32_t Z);
/* forward and backward of loss = mean(((out - target) * 100)^2); gradients
 * replace the previous ones; *loss (host) receives the loss */
int xtc_net_backward(xtc_net *net, const float *fbp, const float *icd, const float *target, int32_t nb, int32_t Y,
                     int32_t X, int32_t Z, double *loss);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8) with the current gradients */
int xtc_net_adam_step(xtc_net *net, float lr);
/* `steps` Adam steps on random py x px x pz patches (batch of them per step)
 * cut from nvol device volume triples (fbp[i], icd[i], target[i], each
 * [Y][X][Z]); losses[step] (host, optional) receives each step's loss. */
int xtc_net_train(xtc_net *net, const float *const *fbp, const float *const *icd, const float *const *target,
                  int32_t nvol, int32_t Y, int32_t X, int32_t Z, int32_t py, int32_t px, int32_t pz, int32_t batch,
                  int32_t steps, float lr, uint64_t seed, float *losses);

/* ---- learned warm start on an engine context (xtg.h) ----------------------
 * The network's inputs are the FBP image (xtg_init_object_fbp) and the
 * multi-resolution start (xtg_init_object_multires with coarse_iters coarse
 * iterations, z halved too when N_z is even and >= 16); its estimate is kept
 * (*used = 1) only if its MAP cost is below the multi-resolution start's by
 * more than 1e-9 relative (both with e = y - Ax - d recomputed; the margin is
 * the noise of the FP64 cost sums); otherwise the multi-resolution start
 * stays (*used = 0) -- the fallback.  ICD then continues at iteration 1.
 * Needs N_x, N_y, N_z multiples of 8. */
struct xtg_ctx;
int xtg_init_object_learned(struct xtg_ctx *ctx, xtc_net *net, int32_t coarse_iters, int32_t *used,
                            double *cost_net, double *cost_base);

#ifdef __cplusplus
}
#endif
#endif
