// xtg_warm.cu -- the learned warm start on an engine context: the FBP image
// and the multi-resolution start go through the network, whose estimate is
// kept only if it lowers the MAP cost.
#include <cstdio>

#include "../../include/xtg.h"
#include "../../include/xtg_cnn.h"

void xtg_set_error_text(const char *msg);
float *xtc_net_start_buffer(xtc_net *n, size_t floats);  // cnn_net.cu
extern "C" int xtg_fbp_image_only(xtg_ctx *c);             // xtg_api.cu
extern "C" int xtg_init_error_model(xtg_ctx *c);           // xtg_api.cu

extern "C" int xtg_init_object_learned(xtg_ctx *ctx, xtc_net *net, int32_t coarse_iters, int32_t *used,
                                       double *cost_net, double *cost_base) {
  if (!ctx || !net || coarse_iters < 0) return XTG_E_ARG;
  int32_t d[11];
  int rc = xtg_dims(ctx, d);
  if (rc) return rc;
  const int N_x = d[0], N_y = d[1], N_z = d[2], N_time = d[3];
  if (N_x % 8 || N_y % 8 || N_z % 8) {
    xtg_set_error_text("xtg_init_object_learned: N_x, N_y and N_z must be multiples of 8");
    return XTG_E_ARG;
  }
  const size_t nvox = (size_t)N_time * N_y * N_x * N_z;
  // the three images live in a buffer the network keeps, so repeated starts
  // on one geometry allocate nothing
  float *buf = xtc_net_start_buffer(net, 3 * nvox);
  if (!buf) {
    xtg_set_error_text("xtg_init_object_learned: out of device memory for the start images");
    return XTG_E_CUDA;
  }
  float *fbp = buf, *icd = buf + nvox, *out = buf + 2 * nvox;
  double ci = 0, cn = 0;
  int use = 0;
  do {
    // the FBP image only: the multi-resolution start below recomputes e
    if ((rc = xtg_fbp_image_only(ctx)) || (rc = xtg_object_to_device(ctx, fbp))) break;
    // the multi-resolution start (it ends with e = y - A delta_t x - d recomputed, so
    // both candidates are costed from a fresh e)
    if ((rc = xtg_init_object_multires(ctx, coarse_iters, N_z % 2 == 0 && N_z >= 16)) ||
        (rc = xtg_object_to_device(ctx, icd)) || (rc = xtg_map_cost_running(ctx, &ci, nullptr, nullptr)))
      break;
    if ((rc = xtc_net_forward(net, fbp, icd, out, N_time, N_y, N_x, N_z))) break;
    if ((rc = xtg_object_from_device(ctx, out)) || (rc = xtg_init_error_model(ctx)) ||
        (rc = xtg_map_cost_running(ctx, &cn, nullptr, nullptr)))
      break;
    // lower by more than the run-to-run noise of the FP64 cost sums (their
    // atomic accumulation order varies), so an unchanged image is not "better"
    use = cn < ci * (1.0 - 1e-9);
    if (!use && ((rc = xtg_object_from_device(ctx, icd)) || (rc = xtg_init_error_model(ctx)))) break;
  } while (0);
  if (rc) return rc;
  if (used) *used = use;
  if (cost_net) *cost_net = cn;
  if (cost_base) *cost_base = ci;
  return 0;
}
