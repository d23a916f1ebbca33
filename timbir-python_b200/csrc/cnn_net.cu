// cnn_net.cu -- the warm-start network: a 3D encoder-decoder (four levels,
// 32/48/64/96 channels, two 3x3x3 convolutions + ReLU per level and side,
// 2x average pooling down, nearest 2x upsampling + skip concatenation up, a
// 1x1 head) mapping (FBP image, image after a few ICD equits) to a residual
// correction of the latter: out = icd + head / scale.  About 1.44 M parameters,
// FP32 master weights, BF16 weights and activations on the tcgen05 tensor
// cores, FP32 gradients, Adam.  All compute runs in this library's kernels;
// the host only sequences launches.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/xtg.h"
#include "../../include/xtg_cnn.h"
#include "xtg_cnn_internal.h"

void xtg_set_error_text(const char *msg);

namespace {

using bf16 = __nv_bfloat16;
constexpr float kScale = 100.f;  // inputs and correction in units of 1/100 per voxel length
constexpr int kLayers = 14;
// (cin as used by the data, cin as stored (multiple of 8), cout)
constexpr int kSpec[kLayers][2] = {{2, 32},  {32, 32}, {32, 48}, {48, 48},  {48, 64}, {64, 64},  {64, 96},
                                   {96, 96}, {160, 64}, {64, 64}, {112, 48}, {48, 48}, {80, 32}, {32, 32}};
constexpr int kHeadC = 32;

int kpad_of(int cin) { return (27 * cin + 63) / 64 * 64; }
int cin_store(int cin_real) { return (cin_real + 7) / 8 * 8; }

struct Layer {
  int cin_real, cin, cout, kpad, kpad_t;
  size_t off_w, off_b;  // offsets in the parameter vector
  bf16 *W = nullptr, *Wt = nullptr;
  bf16 *Wp = nullptr;   // W packed for the tile kernel
  bf16 *Wtp = nullptr;  // Wt packed for the tile kernel (input gradient, layers with cin <= 64)
  bf16 *W64 = nullptr;  // the first layer's W as [cout][64], k = 2 tap + channel
};

struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};

}  // namespace

struct xtc_net {
  Layer L[kLayers];
  size_t n_params = 0, off_hw = 0, off_hb = 0;
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;  // parameters, gradients, Adam moments
  float *graw = nullptr;  // raw weight gradient of the input layer (cin padded)
  double *d_loss = nullptr;
  int *d_err = nullptr;
  int step = 0;
  bool packed = false;
  cudaStream_t st = 0;
  // activations (BF16) and gradients (FP32) for the current batch shape
  int nb = 0, Y = 0, X = 0, Z = 0;
  Buf in0, a[kLayers], u0, u1, u2, p0, p1, p2, g32, gtmp, gskip[3], gpre;
  Buf start;  // the learned start's three images (xtg_warm.cu), kept between calls
};

namespace {

int set_fail(const char *what, cudaError_t e) {
  char b[256];
  snprintf(b, sizeof b, "%s: %s", what, cudaGetErrorString(e));
  xtg_set_error_text(b);
  return XTG_E_CUDA;
}
#define NCK(x)                                   \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) return set_fail(#x, e_); \
  } while (0)

uint64_t mix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double gauss(uint64_t &s) {  // Box-Muller
  const double u1 = ((mix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((mix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

int pack_all(xtc_net *n) {
  for (int i = 0; i < kLayers; i++) {
    Layer &l = n->L[i];
    xtc::pack_weights(l.cin_real, l.cin, l.cout, l.kpad, l.kpad_t, n->P + l.off_w, l.W, i ? l.Wt : nullptr, n->st);
    if (l.Wp) NCK(xtc::conv_tile_pack(l.cin, l.cout, l.kpad, 1, l.W, l.Wp, n->st));
    if (l.Wtp) NCK(xtc::conv_tile_pack(l.cout, l.cin, l.kpad_t, -1, l.Wt, l.Wtp, n->st));
    if (l.W64) NCK(xtc::conv_first_pack(l.cout, l.cin, l.kpad, l.W, l.W64, n->st));
  }
  NCK(cudaGetLastError());
  n->packed = true;
  return 0;
}

int check_err(xtc_net *n) {
  int h = 0;
  NCK(cudaMemcpyAsync(&h, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, n->st));
  NCK(cudaStreamSynchronize(n->st));
  if (h) {
    cudaMemsetAsync(n->d_err, 0, sizeof(int), n->st);
    xtg_set_error_text("xtc_net: tensor-core pipeline wait timed out");
    return XTG_E_TIMEOUT;
  }
  return 0;
}

// activation and gradient buffers for a batch shape
int ensure_buffers(xtc_net *n, int nb, int Y, int X, int Z) {
  if (n->nb == nb && n->Y == Y && n->X == X && n->Z == Z) return 0;
  const size_t v0 = (size_t)nb * Y * X * Z, v1 = v0 / 8, v2 = v1 / 8, v3 = v2 / 8;
  const size_t lv[kLayers] = {v0, v0, v1, v1, v2, v2, v3, v3, v2, v2, v1, v1, v0, v0};
  NCK(n->in0.ensure(v0 * 8 * sizeof(bf16)));
  size_t gmax = 0;
  for (int i = 0; i < kLayers; i++) {
    NCK(n->a[i].ensure(lv[i] * n->L[i].cout * sizeof(bf16)));
    gmax = std::max(gmax, lv[i] * (size_t)n->L[i].cin);
    gmax = std::max(gmax, lv[i] * (size_t)n->L[i].cout);
  }
  NCK(n->p0.ensure(v1 * 32 * sizeof(bf16)));
  NCK(n->p1.ensure(v2 * 48 * sizeof(bf16)));
  NCK(n->p2.ensure(v3 * 64 * sizeof(bf16)));
  NCK(n->u2.ensure(v2 * 160 * sizeof(bf16)));
  NCK(n->u1.ensure(v1 * 112 * sizeof(bf16)));
  NCK(n->u0.ensure(v0 * 80 * sizeof(bf16)));
  NCK(n->g32.ensure(gmax * sizeof(float)));
  NCK(n->gtmp.ensure(gmax * sizeof(float)));
  NCK(n->gpre.ensure(gmax * sizeof(bf16)));
  NCK(n->gskip[0].ensure(v0 * 32 * sizeof(float)));
  NCK(n->gskip[1].ensure(v1 * 48 * sizeof(float)));
  NCK(n->gskip[2].ensure(v2 * 64 * sizeof(float)));
  n->nb = nb;
  n->Y = Y;
  n->X = X;
  n->Z = Z;
  return 0;
}

int conv(xtc_net *n, int li, const bf16 *in, int lvl, bf16 *out) {
  const Layer &l = n->L[li];
  xtc::ConvShape s{n->nb, n->Y >> lvl, n->X >> lvl, n->Z >> lvl, l.cin, l.cout, l.kpad};
  if (l.Wp && xtc::conv_tile_supported(s)) {
    const cudaError_t e = xtc::conv_forward_tile(s, in, l.Wp, n->P + l.off_b, out, 0, 1, n->d_err, n->st);
    if (e != cudaErrorNotSupported) {
      NCK(e);
      return 0;
    }
    cudaGetLastError();
  }
  NCK(xtc::conv_forward(s, in, l.W, n->P + l.off_b, out, 0, 1, n->d_err, n->st));
  return 0;
}

int forward(xtc_net *n, const float *fbp, const float *icd, float *out, const float *target) {
  const int nb = n->nb, Y = n->Y, X = n->X, Z = n->Z;
  const long long v0 = (long long)nb * Y * X * Z;
  cudaStream_t st = n->st;
  bf16 *A[kLayers];
  for (int i = 0; i < kLayers; i++) A[i] = n->a[i].as<bf16>();
  int rc;
  if (target) {  // training keeps the packed input for the first layer's weight gradient
    xtc::pack_input(v0, fbp, icd, kScale, n->in0.as<bf16>(), st);
    if ((rc = conv(n, 0, n->in0.as<bf16>(), 0, A[0]))) return rc;
  } else {
    NCK(xtc::conv_first(nb, Y, X, Z, fbp, icd, kScale, n->L[0].W64, n->P + n->L[0].off_b, n->L[0].cout, A[0],
                        n->d_err, st));
  }
  if ((rc = conv(n, 1, A[0], 0, A[1]))) return rc;
  xtc::avgpool(nb, Y, X, Z, 32, A[1], n->p0.as<bf16>(), st);
  if ((rc = conv(n, 2, n->p0.as<bf16>(), 1, A[2]))) return rc;
  if ((rc = conv(n, 3, A[2], 1, A[3]))) return rc;
  xtc::avgpool(nb, Y / 2, X / 2, Z / 2, 48, A[3], n->p1.as<bf16>(), st);
  if ((rc = conv(n, 4, n->p1.as<bf16>(), 2, A[4]))) return rc;
  if ((rc = conv(n, 5, A[4], 2, A[5]))) return rc;
  xtc::avgpool(nb, Y / 4, X / 4, Z / 4, 64, A[5], n->p2.as<bf16>(), st);
  if ((rc = conv(n, 6, n->p2.as<bf16>(), 3, A[6]))) return rc;
  if ((rc = conv(n, 7, A[6], 3, A[7]))) return rc;
  xtc::up_concat(nb, Y / 4, X / 4, Z / 4, 96, 64, A[7], A[5], n->u2.as<bf16>(), st);
  if ((rc = conv(n, 8, n->u2.as<bf16>(), 2, A[8]))) return rc;
  if ((rc = conv(n, 9, A[8], 2, A[9]))) return rc;
  xtc::up_concat(nb, Y / 2, X / 2, Z / 2, 64, 48, A[9], A[3], n->u1.as<bf16>(), st);
  if ((rc = conv(n, 10, n->u1.as<bf16>(), 1, A[10]))) return rc;
  if ((rc = conv(n, 11, A[10], 1, A[11]))) return rc;
  xtc::up_concat(nb, Y, X, Z, 48, 32, A[11], A[1], n->u0.as<bf16>(), st);
  if ((rc = conv(n, 12, n->u0.as<bf16>(), 0, A[12]))) return rc;
  if ((rc = conv(n, 13, A[12], 0, A[13]))) return rc;
  if (target) NCK(cudaMemsetAsync(n->d_loss, 0, sizeof(double), st));
  xtc::head(v0, kHeadC, A[13], n->P + n->off_hw, n->P + n->off_hb, icd, kScale, out, target, n->d_loss,
            n->g32.as<float>(), n->G + n->off_hw, n->G + n->off_hb, st);
  NCK(cudaGetLastError());
  return 0;
}

// backward of conv li with post-ReLU gradient dpost (FP32) and post-activation
// `post`; writes the input gradient (FP32) to din when din != nullptr
int conv_back(xtc_net *n, int li, const float *dpost, const bf16 *post, const bf16 *in, int lvl, float *din) {
  const Layer &l = n->L[li];
  const long long nv = (long long)n->nb * (n->Y >> lvl) * (n->X >> lvl) * (n->Z >> lvl);
  bf16 *dpre = n->gpre.as<bf16>();
  xtc::relu_back(nv, l.cout, dpost, post, dpre, n->G + l.off_b, n->st);
  xtc::ConvShape s{n->nb, n->Y >> lvl, n->X >> lvl, n->Z >> lvl, l.cin, l.cout, l.kpad};
  if (l.cin == l.cin_real) {
    NCK(xtc::conv_wgrad(s, in, dpre, n->G + l.off_w, n->d_err, n->st));
  } else {
    NCK(cudaMemsetAsync(n->graw, 0, sizeof(float) * 27 * l.cin * l.cout, n->st));
    NCK(xtc::conv_wgrad(s, in, dpre, n->graw, n->d_err, n->st));
    xtc::fold_wgrad(l.cin_real, l.cin, l.cout, n->graw, n->G + l.off_w, n->st);
  }
  if (din) {
    // the input gradient: the same convolution with transposed weights and
    // negated offsets, on the tile kernel where the shape allows
    xtc::ConvShape t{n->nb, n->Y >> lvl, n->X >> lvl, n->Z >> lvl, l.cout, l.cin, l.kpad_t};
    if (l.Wtp && xtc::conv_tile_supported(t)) {
      const cudaError_t e = xtc::conv_forward_tile(t, dpre, l.Wtp, nullptr, din, 2, -1, n->d_err, n->st);
      if (e != cudaErrorNotSupported) {
        NCK(e);
        return 0;
      }
      cudaGetLastError();
    }
    NCK(xtc::conv_forward(t, dpre, l.Wt, nullptr, din, 2, -1, n->d_err, n->st));
  }
  return 0;
}

int backward(xtc_net *n) {
  const int nb = n->nb, Y = n->Y, X = n->X, Z = n->Z;
  cudaStream_t st = n->st;
  bf16 *A[kLayers];
  for (int i = 0; i < kLayers; i++) A[i] = n->a[i].as<bf16>();
  float *g = n->g32.as<float>(), *t = n->gtmp.as<float>();
  float *s0 = n->gskip[0].as<float>(), *s1 = n->gskip[1].as<float>(), *s2 = n->gskip[2].as<float>();
  const size_t v0 = (size_t)nb * Y * X * Z, v1 = v0 / 8, v2 = v1 / 8;
  NCK(cudaMemsetAsync(s0, 0, v0 * 32 * sizeof(float), st));
  NCK(cudaMemsetAsync(s1, 0, v1 * 48 * sizeof(float), st));
  NCK(cudaMemsetAsync(s2, 0, v2 * 64 * sizeof(float), st));
  int rc;
  // decoder, level 0: g = d A13 (from the head)
  if ((rc = conv_back(n, 13, g, A[13], A[12], 0, t))) return rc;                  // t = d A12
  if ((rc = conv_back(n, 12, t, A[12], n->u0.as<bf16>(), 0, g))) return rc;        // g = d u0
  xtc::up_concat_back(nb, Y, X, Z, 48, 32, g, t, s0, st);                          // t = d A11, s0 +=
  if ((rc = conv_back(n, 11, t, A[11], A[10], 1, g))) return rc;                   // g = d A10
  if ((rc = conv_back(n, 10, g, A[10], n->u1.as<bf16>(), 1, t))) return rc;        // t = d u1
  xtc::up_concat_back(nb, Y / 2, X / 2, Z / 2, 64, 48, t, g, s1, st);              // g = d A9, s1 +=
  if ((rc = conv_back(n, 9, g, A[9], A[8], 2, t))) return rc;                      // t = d A8
  if ((rc = conv_back(n, 8, t, A[8], n->u2.as<bf16>(), 2, g))) return rc;          // g = d u2
  xtc::up_concat_back(nb, Y / 4, X / 4, Z / 4, 96, 64, g, t, s2, st);              // t = d A7, s2 +=
  // bottom
  if ((rc = conv_back(n, 7, t, A[7], A[6], 3, g))) return rc;                      // g = d A6
  if ((rc = conv_back(n, 6, g, A[6], n->p2.as<bf16>(), 3, t))) return rc;          // t = d p2
  xtc::avgpool_back(nb, Y / 4, X / 4, Z / 4, 64, t, s2, st);                       // s2 += (d A5 complete)
  // encoder, level 2..0
  if ((rc = conv_back(n, 5, s2, A[5], A[4], 2, g))) return rc;                     // g = d A4
  if ((rc = conv_back(n, 4, g, A[4], n->p1.as<bf16>(), 2, t))) return rc;          // t = d p1
  xtc::avgpool_back(nb, Y / 2, X / 2, Z / 2, 48, t, s1, st);                       // s1 += (d A3 complete)
  if ((rc = conv_back(n, 3, s1, A[3], A[2], 1, g))) return rc;                     // g = d A2
  if ((rc = conv_back(n, 2, g, A[2], n->p0.as<bf16>(), 1, t))) return rc;          // t = d p0
  xtc::avgpool_back(nb, Y, X, Z, 32, t, s0, st);                                   // s0 += (d A1 complete)
  if ((rc = conv_back(n, 1, s0, A[1], A[0], 0, g))) return rc;                     // g = d A0
  if ((rc = conv_back(n, 0, g, A[0], n->in0.as<bf16>(), 0, nullptr))) return rc;
  NCK(cudaGetLastError());
  return 0;
}

int check_dims(int nb, int Y, int X, int Z) {
  if (nb < 1 || Y < 8 || X < 8 || Z < 8 || Y % 8 || X % 8 || Z % 8) {
    xtg_set_error_text("xtc_net: volume dimensions must be positive multiples of 8");
    return XTG_E_ARG;
  }
  return 0;
}

}  // namespace

extern "C" {

int xtc_net_create(uint64_t seed, xtc_net **out) {
  if (!out) return XTG_E_ARG;
  xtc_net *n = new xtc_net();
  size_t off = 0;
  for (int i = 0; i < kLayers; i++) {
    Layer &l = n->L[i];
    l.cin_real = kSpec[i][0];
    l.cin = cin_store(l.cin_real);
    l.cout = kSpec[i][1];
    l.kpad = kpad_of(l.cin);
    l.kpad_t = kpad_of(l.cout);
    l.off_w = off;
    off += (size_t)27 * l.cin_real * l.cout;
    l.off_b = off;
    off += l.cout;
  }
  n->off_hw = off;
  off += kHeadC;
  n->off_hb = off;
  off += 1;
  n->n_params = off;
  std::vector<float> h(off, 0.f);
  uint64_t s = seed;
  for (int i = 0; i < kLayers; i++) {
    const Layer &l = n->L[i];
    const double sd = std::sqrt(2.0 / (27.0 * l.cin_real));  // He initialisation
    for (size_t k = 0; k < (size_t)27 * l.cin_real * l.cout; k++) h[l.off_w + k] = (float)(sd * gauss(s));
  }
  // the head starts at zero: the untrained network returns its ICD input
  cudaError_t e = cudaSuccess;
  auto A = [&](void **p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
  };
  A((void **)&n->P, off * 4);
  A((void **)&n->G, off * 4);
  A((void **)&n->M, off * 4);
  A((void **)&n->V, off * 4);
  A((void **)&n->graw, (size_t)27 * 8 * 32 * 4);
  A((void **)&n->d_loss, 8);
  A((void **)&n->d_err, 4);
  for (int i = 0; i < kLayers; i++) {
    Layer &l = n->L[i];
    A((void **)&l.W, (size_t)l.cout * l.kpad * 2);
    if (i) A((void **)&l.Wt, (size_t)l.cin * l.kpad_t * 2);
    if (l.cout <= 64) A((void **)&l.Wp, xtc::conv_tile_wp_elems(l.cin, l.cout) * 2);
    if (i && l.cin <= 64 && l.cin % 16 == 0) A((void **)&l.Wtp, xtc::conv_tile_wp_elems(l.cout, l.cin) * 2);
    if (i == 0) A((void **)&l.W64, (size_t)l.cout * 64 * 2);
  }
  if (e == cudaSuccess) e = cudaMemcpy(n->P, h.data(), off * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(n->M, 0, off * 4);
  if (e == cudaSuccess) e = cudaMemset(n->V, 0, off * 4);
  if (e == cudaSuccess) e = cudaMemset(n->G, 0, off * 4);
  if (e == cudaSuccess) e = cudaMemset(n->d_err, 0, 4);
  if (e != cudaSuccess) {
    xtc_net_destroy(n);
    return set_fail("xtc_net_create", e);
  }
  *out = n;
  return 0;
}

void xtc_net_destroy(xtc_net *n) {
  if (!n) return;
  for (float *p : {n->P, n->G, n->M, n->V, n->graw})
    if (p) cudaFree(p);
  if (n->d_loss) cudaFree(n->d_loss);
  if (n->d_err) cudaFree(n->d_err);
  for (int i = 0; i < kLayers; i++) {
    if (n->L[i].W) cudaFree(n->L[i].W);
    if (n->L[i].Wt) cudaFree(n->L[i].Wt);
    if (n->L[i].Wp) cudaFree(n->L[i].Wp);
    if (n->L[i].Wtp) cudaFree(n->L[i].Wtp);
    if (n->L[i].W64) cudaFree(n->L[i].W64);
  }
  delete n;
}

int64_t xtc_net_param_count(const xtc_net *n) { return n ? (int64_t)n->n_params : 0; }

int xtc_net_get_params(const xtc_net *n, float *host, int32_t which) {
  if (!n || !host || which < 0 || which > 1) return XTG_E_ARG;
  NCK(cudaStreamSynchronize(n->st));
  NCK(cudaMemcpy(host, which ? n->G : n->P, n->n_params * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int xtc_net_set_params(xtc_net *n, const float *host) {
  if (!n || !host) return XTG_E_ARG;
  NCK(cudaMemcpy(n->P, host, n->n_params * 4, cudaMemcpyHostToDevice));
  n->packed = false;
  return 0;
}

int xtc_net_save(const xtc_net *n, const char *path) {
  if (!n || !path) return XTG_E_ARG;
  std::vector<float> h(n->n_params);
  int rc = xtc_net_get_params(n, h.data(), 0);
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) {
    xtg_set_error_text("xtc_net_save: cannot open the file");
    return XTG_E_ARG;
  }
  const uint32_t hdr[3] = {0x4E435458u /* "XTCN" */, 1u, (uint32_t)n->n_params};
  const bool ok = fwrite(hdr, 4, 3, f) == 3 && fwrite(h.data(), 4, h.size(), f) == h.size();
  fclose(f);
  if (!ok) {
    xtg_set_error_text("xtc_net_save: short write");
    return XTG_E_ARG;
  }
  return 0;
}

int xtc_net_load(xtc_net *n, const char *path) {
  if (!n || !path) return XTG_E_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) {
    xtg_set_error_text("xtc_net_load: cannot open the file");
    return XTG_E_ARG;
  }
  uint32_t hdr[3];
  std::vector<float> h(n->n_params);
  const bool ok = fread(hdr, 4, 3, f) == 3 && hdr[0] == 0x4E435458u && hdr[1] == 1u && hdr[2] == n->n_params &&
                  fread(h.data(), 4, h.size(), f) == h.size();
  fclose(f);
  if (!ok) {
    xtg_set_error_text("xtc_net_load: not a weight file of this network");
    return XTG_E_ARG;
  }
  return xtc_net_set_params(n, h.data());
}

}  // extern "C"

// a device buffer of at least `floats` FP32 values owned by the network and
// kept until it is destroyed (grown when a larger volume asks for more)
float *xtc_net_start_buffer(xtc_net *n, size_t floats) {
  if (!n || n->start.ensure(floats * sizeof(float)) != cudaSuccess) return nullptr;
  return n->start.as<float>();
}

extern "C" {

int xtc_net_forward(xtc_net *n, const float *fbp, const float *icd, float *out, int32_t nb, int32_t Y, int32_t X,
                    int32_t Z) {
  if (!n || !fbp || !icd || !out) return XTG_E_ARG;
  int rc = check_dims(nb, Y, X, Z);
  if (rc) return rc;
  if ((rc = ensure_buffers(n, nb, Y, X, Z))) return rc;
  if (!n->packed && (rc = pack_all(n))) return rc;
  if ((rc = forward(n, fbp, icd, out, nullptr))) return rc;
  return check_err(n);
}

int xtc_net_backward(xtc_net *n, const float *fbp, const float *icd, const float *target, int32_t nb, int32_t Y,
                     int32_t X, int32_t Z, double *loss) {
  if (!n || !fbp || !icd || !target) return XTG_E_ARG;
  int rc = check_dims(nb, Y, X, Z);
  if (rc) return rc;
  if ((rc = ensure_buffers(n, nb, Y, X, Z))) return rc;
  if (!n->packed && (rc = pack_all(n))) return rc;
  NCK(cudaMemsetAsync(n->G, 0, n->n_params * 4, n->st));
  float *scratch = n->gtmp.as<float>();  // the head's output is not kept in training
  if ((rc = forward(n, fbp, icd, scratch, target))) return rc;
  if ((rc = backward(n))) return rc;
  if (loss) NCK(cudaMemcpyAsync(loss, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, n->st));
  return check_err(n);
}

int xtc_net_adam_step(xtc_net *n, float lr) {
  if (!n || !(lr > 0.f)) return XTG_E_ARG;
  n->step++;
  xtc::adam((long long)n->n_params, n->P, n->G, n->M, n->V, lr, 0.9f, 0.999f, 1e-8f, n->step, n->st);
  NCK(cudaGetLastError());
  return pack_all(n);
}

int xtc_net_train(xtc_net *n, const float *const *fbp, const float *const *icd, const float *const *target,
                  int32_t nvol, int32_t Y, int32_t X, int32_t Z, int32_t py, int32_t px, int32_t pz, int32_t batch,
                  int32_t steps, float lr, uint64_t seed, float *losses) {
  if (!n || !fbp || !icd || !target || nvol < 1 || steps < 1 || batch < 1 || py > Y || px > X || pz > Z)
    return XTG_E_ARG;
  int rc = check_dims(batch, py, px, pz);
  if (rc) return rc;
  const size_t pv = (size_t)batch * py * px * pz;
  Buf bf, bi, bt, src, org;
  NCK(bf.ensure(pv * 4));
  NCK(bi.ensure(pv * 4));
  NCK(bt.ensure(pv * 4));
  NCK(src.ensure(3 * (size_t)nvol * sizeof(float *)));
  NCK(org.ensure((size_t)batch * sizeof(int4)));
  std::vector<const float *> hp(3 * (size_t)nvol);
  for (int v = 0; v < nvol; v++) {
    hp[v] = fbp[v];
    hp[nvol + v] = icd[v];
    hp[2 * nvol + v] = target[v];
  }
  NCK(cudaMemcpy(src.p, hp.data(), hp.size() * sizeof(float *), cudaMemcpyHostToDevice));
  const float *const *dsrc = src.as<const float *>();
  uint64_t s = seed;
  std::vector<int4> ho(batch);
  for (int it = 0; it < steps; it++) {
    for (int b = 0; b < batch; b++) {
      ho[b].w = (int)(mix(s) % (uint64_t)nvol);
      ho[b].x = (int)(mix(s) % (uint64_t)(Y - py + 1));
      ho[b].y = (int)(mix(s) % (uint64_t)(X - px + 1));
      ho[b].z = (int)(mix(s) % (uint64_t)(Z - pz + 1));
    }
    NCK(cudaMemcpyAsync(org.p, ho.data(), batch * sizeof(int4), cudaMemcpyHostToDevice, n->st));
    xtc::crop(batch, dsrc, org.as<int4>(), Y, X, Z, py, px, pz, bf.as<float>(), n->st);
    xtc::crop(batch, dsrc + nvol, org.as<int4>(), Y, X, Z, py, px, pz, bi.as<float>(), n->st);
    xtc::crop(batch, dsrc + 2 * nvol, org.as<int4>(), Y, X, Z, py, px, pz, bt.as<float>(), n->st);
    double loss = 0;
    if ((rc = xtc_net_backward(n, bf.as<float>(), bi.as<float>(), bt.as<float>(), batch, py, px, pz, &loss))) return rc;
    if ((rc = xtc_net_adam_step(n, lr))) return rc;
    if (losses) losses[it] = (float)loss;
  }
  NCK(cudaStreamSynchronize(n->st));
  return 0;
}

}  // extern "C"
