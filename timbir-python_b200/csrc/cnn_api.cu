// cnn_api.cu -- C ABI of the warm-start network (include/xtg_cnn.h).
#include <cstdio>

#include "../../include/xtg.h"
#include "../../include/xtg_cnn.h"
#include "xtg_cnn_internal.h"

void xtg_set_error_text(const char *msg);  // xtg_api.cu

namespace {
int *g_err = nullptr;  // device flag: a bounded wait in a tensor-core kernel gave up

int fail(cudaError_t e, const char *what) {
  char b[256];
  snprintf(b, sizeof b, "%s: %s", what, cudaGetErrorString(e));
  xtg_set_error_text(b);
  return XTG_E_CUDA;
}

int check_err_flag(const char *what) {
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, g_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(e, what);
  if (h) {
    cudaMemset(g_err, 0, sizeof(int));
    char b[256];
    snprintf(b, sizeof b, "%s: tensor-core pipeline wait timed out", what);
    xtg_set_error_text(b);
    return XTG_E_TIMEOUT;
  }
  return 0;
}

int ensure_err() {
  if (g_err) return 0;
  cudaError_t e = cudaMalloc(&g_err, sizeof(int));
  if (e != cudaSuccess) return fail(e, "xtc: error flag");
  e = cudaMemset(g_err, 0, sizeof(int));
  return e == cudaSuccess ? 0 : fail(e, "xtc: error flag");
}
}  // namespace

extern "C" {

int xtc_wait_selftest(int32_t arrive, int64_t polls) {
  if (polls < 1) {
    xtg_set_error_text("xtc_wait_selftest: polls must be positive");
    return XTG_E_ARG;
  }
  int rc = ensure_err();
  if (rc) return rc;
  cudaError_t e = xtc::wait_selftest(arrive != 0, (long long)polls, g_err, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(e, "xtc_wait_selftest");
  return check_err_flag("xtc_wait_selftest");
}

int xtc_conv3d_path(const void *in, const void *w, const float *bias, void *out, int32_t nb, int32_t Y, int32_t X,
                    int32_t Z, int32_t cin, int32_t cout, int32_t kpad, int32_t epi, int32_t sign, int32_t path) {
  if (!in || !w || !out || (epi == 0 && !bias) || epi < 0 || epi > 2 || (sign != 1 && sign != -1) ||
      path < XTC_CONV_AUTO || path > XTC_CONV_TILE) {
    xtg_set_error_text("xtc_conv3d: bad argument");
    return XTG_E_ARG;
  }
  int rc = ensure_err();
  if (rc) return rc;
  xtc::ConvShape s{nb, Y, X, Z, cin, cout, kpad};
  const bool tile = path != XTC_CONV_GATHER && xtc::conv_tile_supported(s);
  if (path == XTC_CONV_TILE && !tile) {
    xtg_set_error_text("xtc_conv3d: shape not supported by the tile kernel");
    return XTG_E_ARG;
  }
  cudaError_t e;
  if (tile) {
    // the weights packed per 16-channel chunk, in a buffer kept for later calls
    static void *wp = nullptr;
    static size_t wp_bytes = 0;
    const size_t need = xtc::conv_tile_wp_elems(cin, cout) * 2;
    if (need > wp_bytes) {
      if (wp) cudaFree(wp);
      wp = nullptr;
      wp_bytes = 0;
      if ((e = cudaMalloc(&wp, need)) != cudaSuccess) return fail(e, "xtc_conv3d");
      wp_bytes = need;
    }
    e = xtc::conv_tile_pack(cin, cout, kpad, sign, (const __nv_bfloat16 *)w, (__nv_bfloat16 *)wp, 0);
    if (e == cudaSuccess)
      e = xtc::conv_forward_tile(s, (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)wp, bias, out, epi, sign,
                                 g_err, 0);
  } else {
    e = xtc::conv_forward(s, (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)w, bias, out, epi, sign, g_err, 0);
  }
  if (e != cudaSuccess) return fail(e, "xtc_conv3d");
  e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return fail(e, "xtc_conv3d");
  return check_err_flag("xtc_conv3d");
}

int xtc_conv3d(const void *in, const void *w, const float *bias, void *out, int32_t nb, int32_t Y, int32_t X,
               int32_t Z, int32_t cin, int32_t cout, int32_t kpad, int32_t epi, int32_t sign) {
  return xtc_conv3d_path(in, w, bias, out, nb, Y, X, Z, cin, cout, kpad, epi, sign, XTC_CONV_AUTO);
}

int xtc_conv3d_wgrad(const void *in, const void *dout, float *dw, int32_t nb, int32_t Y, int32_t X, int32_t Z,
                     int32_t cin, int32_t cout) {
  return xtc_conv3d_wgrad_path(in, dout, dw, nb, Y, X, Z, cin, cout, XTC_CONV_AUTO);
}

int xtc_conv3d_wgrad_path(const void *in, const void *dout, float *dw, int32_t nb, int32_t Y, int32_t X, int32_t Z,
                          int32_t cin, int32_t cout, int32_t path) {
  if (!in || !dout || !dw || path < XTC_CONV_AUTO || path > XTC_CONV_TILE) {
    xtg_set_error_text("xtc_conv3d_wgrad: bad argument");
    return XTG_E_ARG;
  }
  int rc = ensure_err();
  if (rc) return rc;
  xtc::ConvShape s{nb, Y, X, Z, cin, cout, 0};
  if (path == XTC_CONV_TILE && !xtc::wgrad_tile_supported(s)) {
    xtg_set_error_text("xtc_conv3d_wgrad: shape not supported by the tile kernel");
    return XTG_E_ARG;
  }
  cudaError_t e = xtc::conv_wgrad(s, (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)dout, dw, g_err, 0, path);
  if (e != cudaSuccess) return fail(e, "xtc_conv3d_wgrad");
  e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return fail(e, "xtc_conv3d_wgrad");
  return check_err_flag("xtc_conv3d_wgrad");
}

}  // extern "C"
