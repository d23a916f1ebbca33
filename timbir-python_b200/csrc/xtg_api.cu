// xtg_api.cu -- libxtgpu: device buffers, the non-ICD kernels and the C ABI
// declared in include/xtg.h.
//
// Kernels here (all HBM-bound integer/float streaming, no tensor cores):
//   k_amatrix_batch   A-matrix columns (calcAMatrixColumnforAngle) for a list
//   k_fp<MODE>        forward projection as a gather: one warp per (view, bin),
//                     lanes over detector rows, candidate columns evaluated 32 at a
//                     time and accumulated in the reference's (row, col) order
//                     (FP32 = bit-exact with initErrorSinogam; FP64 = resync/cost)
//   k_prior_cost64    qGGMRF prior over forward neighbour pairs, FP64
//   k_running_cost64  data term from the running e, FP64
//   k_zinger_refresh  ProjSelect = |e sqrt(w)| < T
//   k_vsc_filter / k_rs_hist + k_rs_pick / k_nhicd_compact   NHICD selection
//   k_radix_select    the same order statistic in one CTA (allocation-free path)
//   k_offset_* / k_var_*   offset d and variance re-estimation
//   k_build_items / k_magsum / k_build_a16 / k_counts / object transposes
#include <algorithm>
#include <numeric>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/xtg.h"
#include "xtg_internal.h"

using namespace xtg;

static thread_local char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// error text from the warm-start network's entry points (cnn_api.cu)
void xtg_set_error_text(const char *msg) { snprintf(g_err, sizeof g_err, "%s", msg); }

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      set_err("CUDA error %s at %s:%d: %s", cudaGetErrorName(e_), __FILE__, __LINE__,        \
              cudaGetErrorString(e_));                                                       \
      return XTG_E_CUDA;                                                                     \
    }                                                                                        \
  } while (0)

#define NSLOT 64
// parallel ICD: at most 1 in XTG_CONC_DIV of the columns updated at once
#define XTG_CONC_DIV 32
// ICD footprint loads keep w in L2 (like e) when e and w together take at
// most XTG_W_KEEP_BYTES; larger sinograms evict w first
#ifndef XTG_W_KEEP
#define XTG_W_KEEP 1
#endif
#ifndef XTG_W_KEEP_BYTES
#define XTG_W_KEEP_BYTES (48u << 20)
#endif

struct RsState;  // radix-select state per segment (defined with its kernels)

struct xtg_ctx {
  xt_params prm;
  xt_geom g;
  xt_views v;
  DevGeo G;
  std::vector<float> hr;
  std::vector<int> mcols, col_rank;
  int n_masked = 0;
  size_t ns = 0, nrt = 0, nvox = 0, nmag = 0, nxy = 0;
  int vmax = 0;
  // device arrays
  float *d_y = nullptr, *d_w = nullptr, *d_e = nullptr, *d_d = nullptr, *d_x = nullptr, *d_mag = nullptr;
  float *d_hr = nullptr, *d_cos = nullptr, *d_sin = nullptr, *d_ax = nullptr, *d_filt = nullptr, *d_tmp = nullptr;
  float *d_num = nullptr, *d_den = nullptr, *d_thr = nullptr, *d_var = nullptr;
  int *d_view_idx = nullptr, *d_view_start = nullptr, *d_view_num = nullptr, *d_fov = nullptr;
  int *d_mcols = nullptr, *d_rank = nullptr, *d_counter = nullptr, *d_nhcnt = nullptr, *d_err = nullptr;
  int *d_kth = nullptr;
  unsigned *d_rs_hist = nullptr;  // [segments][256] radix-select histograms
  RsState *d_rs_st = nullptr;     // [segments]
  int4 *d_items = nullptr, *d_nh = nullptr;
  size_t items_cap = 0, nh_cap = 0;
  double *d_red = nullptr;       // [8][NSLOT] reduction slots
  double *d_absx = nullptr;      // [NSLOT]
  unsigned long long *d_cnt = nullptr;  // [4]
  // A column table (CSC): entry runs per (frame, masked column)
  long long *d_tstart = nullptr;
  int *d_toff = nullptr;
  float *d_tval32 = nullptr, *d_tscale = nullptr;
  __half *d_tval16 = nullptr;
  int table_mode = 0;  // 0 none, XTG_A_FP16 or XTG_A_TABLE32 when built
  // bin-major A table of the projector (rows (view, bin)); csr_state 0 = not
  // tried yet, 1 = built, -1 = not used (does not fit, or the gather projector
  // was requested)
  long long *d_cptr = nullptr;
  int2 *d_cent = nullptr;
  int csr_state = 0, projector = XTG_PROJ_AUTO;
  long long csr_nnz = 0;
  long long table_nnz = 0;
  int table_max = 0;
  // options
  int a_mode = XTG_A_FP32, order = XTG_ORDER_PARALLEL, max_columns = 0, span = 3;
  unsigned long long seed = 0x5eed5eedULL;
  int sm_count = 0;
  long long l2_bytes = 0;
  std::vector<double> t_in, a_in;  // view times / angles as given (for the coarse context)
  xtg_ctx *coarse = nullptr;      // multi-resolution start: the 2x coarser grid
  int coarse_flags = 0;           // the XTG_MULTIRES_* flags it was built for
  int zslab_req = 0;  // z slices per ICD work piece; 0 = from the L2 size
  // z slab of a volume split over processes (xtg_set_slab): caller-owned
  // device planes [N_time][N_y][N_x] and the exchange hook
  float *send_lo = nullptr, *send_hi = nullptr;
  const float *halo_lo = nullptr, *halo_hi = nullptr;
  xtg_exchange_fn xfn = nullptr;
  void *xuser = nullptr;
  int xphase = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st_copy = nullptr;               // host-to-device copies that overlap the projector
  cudaEvent_t ev_y = nullptr, ev_w = nullptr;  // ... and their completion on it
  // asynchronous object download: the transposed copy in d_dl leaves on
  // st_copy after ev_dx; ev_dl marks its arrival on the host
  float *d_dl = nullptr;
  cudaEvent_t ev_dx = nullptr, ev_dl = nullptr;
  int dl_pending = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ek0 = nullptr, ek1 = nullptr;
  std::vector<cudaEvent_t> tev;  // start/stop pairs of the ICD launches of one iteration
  int have_sino = 0;
  long long launches = 0;
  float last_kms = 0.f;
  long long last_items = 0, last_icd = 0;
  long long icd_launches = 0;  // ICD column-kernel launches since creation
  size_t dev_bytes = 0;
  // Park-Miller state for the reference-order mode (randlib.c:119-168)
  unsigned int sd[2] = {0, 0};
  long rtmp = 0;
};

// ------------------------------------------------------------- helpers --
template <typename T>
static int dalloc(xtg_ctx *c, T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    set_err("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return XTG_E_CUDA;
  }
  c->dev_bytes += n * sizeof(T);
  return 0;
}

static unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

static void rng_seed(xtg_ctx *c, unsigned int s) {
  c->rtmp = s;
  c->sd[0] = (unsigned)(c->rtmp >> 16);
  c->sd[1] = (unsigned)(c->rtmp & 0xffff);
}
static double rng_next(xtg_ctx *c) {
  c->sd[1] *= 16807u;
  c->sd[0] *= 16807u;
  c->rtmp = (long)((c->sd[0] >> 15) + ((c->sd[0] & 0x7fff) << 16));
  c->rtmp += (long)c->sd[1];
  if (c->rtmp & 0x80000000L) {
    c->rtmp++;
    c->rtmp &= 0x7fffffffL;
  }
  c->sd[0] = (unsigned)(c->rtmp >> 16);
  c->sd[1] = (unsigned)(c->rtmp & 0xffff);
  return ((double)c->rtmp) / 2147483647.0;
}

// ------------------------------------------------------------- kernels --
__global__ void k_amatrix_batch(DevGeo G, const float *hr, const float *cosv, const float *sinv, int n,
                                const int *rows, const int *cols, const int *views, float *vals, int *idx, int *cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = views[i];
  float v[XT_AMAX];
  int first;
  const int m = xt_amatrix_view(G, hr + (size_t)p * XT_HR_STRIDE, cosv[p], sinv[p], rows[i], cols[i], v, &first);
  // report the reference's (value, index) list: drop zero slots of the dense run
  int k = 0;
  for (int s = 0; s < m; s++)
    if (v[s] > 0.f) {
      vals[(size_t)i * G.amax + k] = v[s];
      idx[(size_t)i * G.amax + k] = first + s;
      k++;
    }
  cnt[i] = k;
}

// qGGMRF prior over forward neighbour pairs (XT_ICD_update.c:202-294), FP64.
// halo_hi (z slab with a neighbour above): the pairs from the top slice into
// that neighbour's bottom slice belong to this slab's sum, as the reference's
// ranks other than the last include Object[i][N_z+1] (XT_ICD_update.c:203-205).
__global__ void __launch_bounds__(256, 3) k_prior_cost64(DevGeo G, const float *x, const float *halo_hi, double *slots) {
  // one warp per z-line (f, j, k), lanes over z: the line's coordinates are
  // decoded once, every load is a coalesced run of the line
  const long long nlines = (long long)G.N_time * G.N_y * G.N_x;
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  // rho(d) = (d^2 / sq) / (c + |d|^(2-p) / sqp) evaluated as
  // d^2 / (sq c + (sq / sqp) 2^((2-p) log2 |d|)): one division, and
  // log2 / exp2 in place of pow (the same value to a few ulp)
  const double ks1 = (double)G.Sigma_S_Q * G.C_S, ks2 = (double)G.Sigma_S_Q / G.Sigma_S_Q_P;
  const double kt1 = (double)G.Sigma_T_Q * G.C_T, kt2 = (double)G.Sigma_T_Q / G.Sigma_T_Q_P;
  const double e2p = 2.0 - (double)G.MRF_P;
  auto rho = [&](double d, double k1, double k2) -> double {
    const double a = fabs(d);
    return a == 0.0 ? 0.0 : (a * a) / (k1 + k2 * exp2(e2p * log2(a)));
  };
  const size_t plane = (size_t)G.N_y * G.N_x;
  double acc = 0.0;
  for (long long L = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); L < nlines; L += nwarps) {
    const int k = (int)(L % G.N_x);
    const long long r = L / G.N_x;
    const int j = (int)(r % G.N_y);
    const int f = (int)(r / G.N_y);
    const float *xl = x + (size_t)L * G.N_z;
    for (int z = lane; z < G.N_z; z += 32) {
      const double v = xl[z];
      auto term = [&](int dz, int dy, int dx) {
        const int jj = j + dy, kk = k + dx, zz = z + dz;
        if (jj < 0 || jj >= G.N_y || kk < 0 || kk >= G.N_x || (zz >= G.N_z && !halo_hi)) return;
        const long long off = (long long)dy * G.N_x + dx;
        const double u = zz == G.N_z ? (double)halo_hi[(size_t)(L + off)] : (double)xl[off * G.N_z + zz];
        acc += (double)G.SF[(1 + dz) * 9 + (1 + dy) * 3 + (1 + dx)] * rho(v - u, ks1, ks2);
      };
      term(0, 0, 1);
      term(0, 1, -1);
      term(0, 1, 0);
      term(0, 1, 1);
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) term(1, dy, dx);
      if (f + 1 < G.N_time)
        acc += (double)G.TF * rho(v - (double)xl[plane * G.N_z + z], kt1, kt2);
    }
  }
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
    atomicAdd(&slots[blockIdx.x % NSLOT], s);
  }
}

// data term from the running e (XT_ICD_update.c:188-200), FP64 arithmetic.
// boundary slices of this slab for its neighbours: lo = slice 0, hi = slice
// N_z - 1, each [N_time][N_y][N_x]
__global__ void k_slab_pack(DevGeo G, const float *x, float *lo, float *hi) {
  const size_t n = (size_t)G.N_time * G.N_y * G.N_x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    if (lo) lo[q] = x[q * G.N_z];
    if (hi) hi[q] = x[q * G.N_z + G.N_z - 1];
  }
}

// generalized-Huber data term of one entry (XT_ICD_update.c:192-198), FP64
__device__ __forceinline__ double huber_term(float e, float w, double T, double delta) {
  const double s = (double)e * sqrt((double)w);
  return fabs(s) < T ? s * s : 2.0 * delta * T * fabs(s) + T * T * (1.0 - 2.0 * delta);
}

// Data term of the running e (FP64 sums).  n4 = n / 4 entries are read as
// float4 (16-byte loads, two in flight per thread), the rest one by one.
__global__ void k_running_cost64(size_t n, const float *e, const float *w, float T, float delta, double *slots) {
  const double Td = T, dd = delta;
  double acc = 0.0;
  const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
  const float4 *e4 = reinterpret_cast<const float4 *>(e), *w4 = reinterpret_cast<const float4 *>(w);
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + stride < n4; i += 2 * stride) {
    const float4 ea = __ldcs(e4 + i), wa = __ldcs(w4 + i), eb = __ldcs(e4 + i + stride), wb = __ldcs(w4 + i + stride);
    acc += huber_term(ea.x, wa.x, Td, dd) + huber_term(ea.y, wa.y, Td, dd) + huber_term(ea.z, wa.z, Td, dd) +
           huber_term(ea.w, wa.w, Td, dd);
    acc += huber_term(eb.x, wb.x, Td, dd) + huber_term(eb.y, wb.y, Td, dd) + huber_term(eb.z, wb.z, Td, dd) +
           huber_term(eb.w, wb.w, Td, dd);
  }
  for (; i < n4; i += stride) {
    const float4 ea = __ldcs(e4 + i), wa = __ldcs(w4 + i);
    acc += huber_term(ea.x, wa.x, Td, dd) + huber_term(ea.y, wa.y, Td, dd) + huber_term(ea.z, wa.z, Td, dd) +
           huber_term(ea.w, wa.w, Td, dd);
  }
  for (size_t q = 4 * n4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
    acc += huber_term(e[q], w[q], Td, dd);
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
    atomicAdd(&slots[blockIdx.x % NSLOT], s);
  }
}

// ProjSelect = |e sqrt(w)| < T, in double like the reference's mixed
// expression; float4 loads for the first n / 4 * 4 entries.
__device__ __forceinline__ unsigned char zsel(float e, float w, double T) {
  return (fabs((double)e * sqrt((double)w)) < T) ? 1 : 0;
}
__global__ void k_zinger_refresh(size_t n, const float *e, const float *w, float T, unsigned char *sel,
                                 unsigned long long *count) {
  const double Td = T;
  unsigned c = 0;
  const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
  const float4 *e4 = reinterpret_cast<const float4 *>(e), *w4 = reinterpret_cast<const float4 *>(w);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const float4 ea = __ldcs(e4 + i), wa = __ldcs(w4 + i);
    const unsigned char s0 = zsel(ea.x, wa.x, Td), s1 = zsel(ea.y, wa.y, Td), s2 = zsel(ea.z, wa.z, Td),
                        s3 = zsel(ea.w, wa.w, Td);
    if (sel) reinterpret_cast<uchar4 *>(sel)[i] = make_uchar4(s0, s1, s2, s3);
    c += s0 + s1 + s2 + s3;
  }
  for (size_t q = 4 * n4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const unsigned char s = zsel(e[q], w[q], Td);
    if (sel) sel[q] = s;
    c += s;
  }
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// ComputeVSC (XT_NHICD.c:128-162): 5x5 Hamming-weighted sum, summed in the
// reference's order in FP32.
__constant__ float c_vsc[25] = {0.0064f, 0.0432f, 0.0800f, 0.0432f, 0.0064f, 0.0432f, 0.2916f, 0.5400f, 0.2916f,
                                0.0432f, 0.0800f, 0.5400f, 1.0000f, 0.5400f, 0.0800f, 0.0432f, 0.2916f, 0.5400f,
                                0.2916f, 0.0432f, 0.0064f, 0.0432f, 0.0800f, 0.0432f, 0.0064f};

__global__ void k_vsc_filter(int nseg, int ny, int nx, const float *map, float *out) {
  const size_t n = (size_t)nseg * ny * nx;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(q % nx);
    const int j = (int)((q / nx) % ny);
    const size_t seg = q / ((size_t)nx * ny);
    const float *m = map + seg * (size_t)nx * ny;
    float f = 0.f;
    for (int p = -2; p <= 2; p++)
      for (int s = -2; s <= 2; s++)
        if (j + p >= 0 && j + p < ny && k + s >= 0 && k + s < nx)
          f = __fadd_rn(f, __fmul_rn(c_vsc[(p + 2) * 5 + s + 2], m[(size_t)(j + p) * nx + (k + s)]));
    out[q] = f;
  }
}

// k-th smallest (1-based) of each segment by 4 passes of 8-bit radix
// histograms; the exact order statistic RandomizedSelect returns
// (XT_NHICD.c:63-126).
__global__ void __launch_bounds__(1024) k_radix_select(const float *vals, int seglen, const int *kth, float *out) {
  __shared__ unsigned hist[256];
  __shared__ unsigned s_prefix, s_mask, s_k;
  const float *v = vals + (size_t)blockIdx.x * seglen;
  if (threadIdx.x == 0) {
    s_prefix = 0;
    s_mask = 0;
    s_k = (unsigned)kth[blockIdx.x];
  }
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const unsigned pre = s_prefix, msk = s_mask;
    for (int i = threadIdx.x; i < seglen; i += blockDim.x) {
      const unsigned key = xt_f2key(v[i]);
      if ((key & msk) == pre) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned k = s_k, cum = 0;
      int b = 0;
      for (; b < 255; b++) {
        if (cum + hist[b] >= k) break;
        cum += hist[b];
      }
      s_k = k - cum;
      s_prefix = pre | ((unsigned)b << shift);
      s_mask = msk | (255u << shift);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = xt_key2f(s_prefix);
}

// The same order statistic spread over many CTAs per segment: per 8-bit pass,
// k_rs_hist counts the keys that match the prefix found so far into a global
// 256-bin histogram of the segment (a warp whose lanes share one bin adds 32
// with a single atomic), and k_rs_pick finds the bin that holds the k-th key,
// narrows the prefix and clears the histogram for the next pass.
struct RsState {
  unsigned prefix, mask, k, pad;
};

__global__ void k_rs_init(const int *kth, RsState *st, unsigned *hist) {
  if (threadIdx.x == 0) st[blockIdx.x] = RsState{0u, 0u, (unsigned)kth[blockIdx.x], 0u};
  for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[(size_t)blockIdx.x * 256 + b] = 0u;
}

__global__ void __launch_bounds__(256) k_rs_hist(const float *vals, int seglen, int shift, const RsState *st,
                                                 unsigned *hist) {
  __shared__ unsigned h[256];
  const int seg = blockIdx.y, lane = threadIdx.x & 31;
  h[threadIdx.x] = 0u;
  __syncthreads();
  const unsigned pre = st[seg].prefix, msk = st[seg].mask;
  const float *v = vals + (size_t)seg * seglen;
  const int stride = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x - lane; i0 < seglen; i0 += stride) {
    const int i = i0 + lane;
    unsigned bin = 256u;  // no key here, or not under the prefix
    if (i < seglen) {
      const unsigned key = xt_f2key(v[i]);
      if ((key & msk) == pre) bin = (key >> shift) & 255u;
    }
    const unsigned b0 = __shfl_sync(0xffffffffu, bin, 0);
    if (__all_sync(0xffffffffu, bin == b0)) {
      if (lane == 0 && b0 < 256u) atomicAdd(&h[b0], 32u);
    } else if (bin < 256u) {
      atomicAdd(&h[bin], 1u);
    }
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[(size_t)seg * 256 + threadIdx.x], h[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_rs_pick(int shift, RsState *st, unsigned *hist, float *out) {
  const int seg = blockIdx.x;
  unsigned *hs = hist + (size_t)seg * 256;
  if (threadIdx.x == 0) {
    const unsigned k = st[seg].k;
    unsigned cum = 0;
    int b = 0;
    for (; b < 255; b++) {
      if (cum + hs[b] >= k) break;
      cum += hs[b];
    }
    st[seg].k = k - cum;
    st[seg].prefix |= (unsigned)b << shift;
    st[seg].mask |= 255u << shift;
    if (shift == 0) out[seg] = xt_key2f(st[seg].prefix);
  }
  __syncthreads();
  hs[threadIdx.x] = 0u;
}

// columns above the threshold -> NHICD work items.  List 0 holds the
// (frame, block) pairs the reference updates in its first half-pass (block
// parity = frame parity, XT_ICD_update.c:846-857), list 1 the others.
// A selected column outside the object-support disk has no voxel to update;
// the reference still visits it, which only zeroes its MagUpdateMap entry
// (XT_VoxUpdate.c:128, 138), so that is all done for it here.
__global__ void k_nhicd_compact(int ntime, int nzb, int ny, int nx, const float *filt, const float *thr,
                                const int *col_rank, float *mag, int4 *list0, int4 *list1, int *cnt, int cap0,
                                int cap1) {
  const size_t n = (size_t)ntime * nzb * ny * nx;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t seg = q / ((size_t)nx * ny);
    if (!(filt[q] > thr[seg])) continue;
    const int k = (int)(q % nx), j = (int)((q / nx) % ny);
    if (col_rank[(size_t)j * nx + k] < 0) {
      mag[q] = 0.f;
      continue;
    }
    const int b = (int)(seg % nzb), f = (int)(seg / nzb);
    const int h = ((f & 1) == (b & 1)) ? 0 : 1;
    const int slot = atomicAdd(&cnt[h], 1);
    if (h == 0) {
      if (slot < cap0) list0[slot] = make_int4(f, j, k, b);
    } else {
      if (slot < cap1) list1[slot] = make_int4(f, j, k, b);
    }
  }
}

__global__ void k_clamp_count(int *cnt, int cap0, int cap1) {
  if (threadIdx.x == 0) {
    cnt[0] = min(cnt[0], cap0);
    cnt[1] = min(cnt[1], cap1);
  }
}

// update_Sinogram_Offset (XT_ICD_update.c:666-759), one thread per (r, t),
// views summed in order; FP32 like the reference, sums for gamma in FP64.
__global__ void k_offset_numden(DevGeo G, const float *e, const float *w, const float *d, float *num, float *den,
                                double *sums) {
  const int nrt = G.N_r * G.N_t;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0, b = 0;
  if (q < nrt) {
    float nm = 0.f, dn = 0.f;
    const float td = G.T * G.delta;
    for (int p = 0; p < G.N_p; p++) {
      const size_t s = (size_t)p * nrt + q;
      const float ev = e[s], wv = w[s];
      const float temp = (float)((double)td * sqrt((double)wv));
      if (fabs((double)ev * sqrt((double)wv)) < (double)G.T) {
        nm = __fadd_rn(nm, __fmul_rn(ev, wv));
        dn = __fadd_rn(dn, wv);
      } else {
        const float sign = (float)((ev > 0.f) - (ev < 0.f));
        nm = __fadd_rn(nm, __fmul_rn(temp, sign));
        dn = (float)((double)dn + (double)temp / fabs((double)ev));
      }
    }
    num[q] = nm;
    den[q] = dn;
    a = (double)d[q] + (double)nm / (double)dn;
    b = 1.0 / (double)dn;
  }
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, off);
    b += __shfl_xor_sync(0xffffffffu, b, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], a);
    atomicAdd(&sums[1], b);
  }
}

__global__ void k_offset_apply(DevGeo G, float *e, float *d, const float *num, const float *den, const double *sums,
                               int zero_mean) {
  const int nrt = G.N_r * G.N_t;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrt) return;
  const float gamma = zero_mean ? (float)(sums[0] / sums[1]) : 0.f;
  const float corr = __fdiv_rn(__fsub_rn(num[q], gamma), den[q]);
  d[q] = __fadd_rn(d[q], corr);
  for (int p = 0; p < G.N_p; p++) {
    const size_t s = (size_t)p * nrt + q;
    e[s] = __fsub_rn(e[s], corr);
  }
}

// update_variance_parameter (XT_ICD_update.c:633-664): w *= var, sum the
// data term (the zinger branch uses sqrt(w * var) after that product, as the
// reference does), then var = sum / N and w /= var.
__global__ void k_var_sum(size_t n, const float *e, float *w, const float *var, float T, float delta, double *slots) {
  double acc = 0.0;
  const float vv = *var;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float w0 = w[i];
    const bool sel = fabs((double)e[i] * sqrt((double)w0)) < (double)T;
    const float w1 = __fmul_rn(w0, vv);
    w[i] = w1;
    if (sel)
      acc += (double)__fmul_rn(__fmul_rn(e[i], e[i]), w1);
    else
      acc += fabs((double)e[i]) * (double)delta * (double)T * sqrt((double)__fmul_rn(w1, vv));
  }
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
    atomicAdd(&slots[blockIdx.x % NSLOT], s);
  }
}

__global__ void k_var_finish(const double *slots, double n, float *var) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < NSLOT; q++) s += slots[q];
    *var = (float)(s / n);
  }
}

__global__ void k_scale_weights(size_t n, float *w, const float *var) {
  const float vv = *var;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    w[i] = __fdiv_rn(w[i], vv);
}

// [N_time][N_z][N_y][N_x] <-> [N_time][N_y][N_x][N_z]
__global__ void k_obj_h2d(DevGeo G, const float *src, float *dst) {
  const size_t n = (size_t)G.N_time * G.N_z * G.N_y * G.N_x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % G.N_x);
    size_t r = i / G.N_x;
    const int j = (int)(r % G.N_y);
    r /= G.N_y;
    const int z = (int)(r % G.N_z);
    const size_t f = r / G.N_z;
    dst[((f * G.N_y + j) * G.N_x + k) * G.N_z + z] = src[i];
  }
}
__global__ void k_obj_d2h(DevGeo G, const float *src, float *dst) {
  const size_t n = (size_t)G.N_time * G.N_z * G.N_y * G.N_x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % G.N_x);
    size_t r = i / G.N_x;
    const int j = (int)(r % G.N_y);
    r /= G.N_y;
    const int z = (int)(r % G.N_z);
    const size_t f = r / G.N_z;
    dst[i] = src[((f * G.N_y + j) * G.N_x + k) * G.N_z + z];
  }
}

// random visiting order of every (frame, masked column) whole z-line
__global__ void k_build_items(int n, int n_masked, int nx, const int *mcols, unsigned long long key, int4 *items) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int v = (int)xt_perm((uint32_t)q, (uint32_t)n, key);
  const int f = v / n_masked, c = mcols[v % n_masked];
  items[q] = make_int4(f, c / nx, c % nx, -1);
}

// sum of MagUpdateMap over the random lists (XT_ICD_update.c:889-894)
__global__ void k_magsum(DevGeo G, int n_masked, const int *mcols, const float *mag, double *slots) {
  const size_t n = (size_t)G.N_time * G.nzb * n_masked;
  double acc = 0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t seg = q / n_masked;
    acc += (double)mag[seg * (size_t)G.N_y * G.N_x + mcols[q % n_masked]];
  }
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
    atomicAdd(&slots[blockIdx.x % NSLOT], s);
  }
}

// genSinogram_subsampleCounts (XT_genSinogram.c:303-374)
__global__ void k_counts(DevGeo G, int mxy, int mz, const float *bright, const float *counts, float bh, float *y,
                         float *w) {
  const size_t n = (size_t)G.N_p * G.N_r * G.N_t;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(q % G.N_t);
    const int r = (int)((q / G.N_t) % G.N_r);
    const size_t p = q / ((size_t)G.N_t * G.N_r);
    const int Rr = G.N_r * mxy, Tt = G.N_t * mz;
    float wt = 0.f, bt = 0.f;
    for (int a = 0; a < mxy; a++)
      for (int b = 0; b < mz; b++) {
        wt = __fadd_rn(wt, counts[(p * Rr + (size_t)(r * mxy + a)) * Tt + (t * mz + b)]);
        bt = __fadd_rn(bt, bright[(size_t)(r * mxy + a) * Tt + (t * mz + b)]);
      }
    const float tmp = (float)log((double)__fdiv_rn(bt, wt));
    y[q] = (float)((double)bh * tmp * tmp + tmp);
    w[q] = wt;
  }
}

__global__ void k_fill(size_t n, float *p, float v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

// ------------------------------------------------------------ host side --
static DevGeo make_devgeo(const xt_geom &g, int positivity) {
  DevGeo G;
  memset(&G, 0, sizeof(G));
  G.N_r = g.N_r; G.N_t = g.N_t; G.N_p = g.N_p; G.N_x = g.N_x; G.N_y = g.N_y; G.N_z = g.N_z;
  G.N_time = g.N_time; G.zovl = g.zovl; G.nzb = g.nzb; G.zstep = g.zstep; G.amax = g.amax;
  G.positivity = positivity;
  G.delta_r = g.delta_r; G.delta_t = g.delta_t; G.R0 = g.R0; G.RMax = g.RMax; G.x0 = g.x0; G.y0 = g.y0;
  G.delta_xy = g.delta_xy; G.OffsetR = g.OffsetR; G.MRF_P = g.MRF_P; G.C_S = g.C_S; G.C_T = g.C_T;
  G.alpha = g.alpha; G.Sigma_S_Q = g.Sigma_S_Q; G.Sigma_S_Q_P = g.Sigma_S_Q_P; G.Sigma_T_Q = g.Sigma_T_Q;
  G.Sigma_T_Q_P = g.Sigma_T_Q_P;
  for (int i = 0; i < 27; i++) G.SF[i] = g.SF[i];
  G.TF = g.TF; G.T = g.T; G.delta = g.delta;
  return G;
}

static double fp_win_margin(const xtg_ctx *c) { return 1e-4 * (double)c->g.N_r * c->g.delta_r + 1e-3 * c->g.delta_r; }

// The projector's bin-major A table, built at the first projection of the
// context when it fits in free device memory next to the column table the
// ICD kernel may still build (and 2 GiB to spare); otherwise the projector
// evaluates A on the fly (k_fp_bins).  Only CUDA errors are returned.
static cudaError_t ensure_csr(xtg_ctx *c) {
  if (c->csr_state) return cudaSuccess;
  c->csr_state = -1;
  if (c->projector == XTG_PROJ_GATHER) return cudaSuccess;
  // entries hold a z-line's element offset within its frame as an int32
  if ((size_t)c->g.N_y * c->g.N_x * c->g.N_z >= ((size_t)1 << 31)) return cudaSuccess;
  const size_t rows = (size_t)c->g.N_p * c->g.N_r;
  int *d_cnt = nullptr;
  if (cudaMalloc(&d_cnt, rows * 4) != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  CsrBuildArgs B;
  memset(&B, 0, sizeof(B));
  B.hr = c->d_hr; B.cosv = c->d_cos; B.sinv = c->d_sin; B.win_margin = fp_win_margin(c); B.count = d_cnt;
  cudaError_t e = launch_csr_build(c->G, B, 0, c->span, c->st);
  std::vector<int> cnt(rows);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), d_cnt, rows * 4, cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(d_cnt);
  c->launches++;
  if (e != cudaSuccess) return e;
  std::vector<long long> ptr(rows + 1, 0);
  for (size_t i = 0; i < rows; i++) ptr[i + 1] = ptr[i] + cnt[i];
  const long long nnz = ptr[rows];
  size_t fr = 0, tot = 0;
  if ((e = cudaMemGetInfo(&fr, &tot)) != cudaSuccess) return e;
  // the column table, if one is still to be built, has at most as many entries
  const size_t pending = (c->a_mode != XTG_A_FP32 && c->table_mode == 0) ? (size_t)nnz * 8 : 0;
  const size_t need = (size_t)nnz * 8 + (rows + 1) * 8;
  if (need + pending + ((size_t)2 << 30) > fr) return cudaSuccess;
  if (cudaMalloc(&c->d_cptr, (rows + 1) * 8) != cudaSuccess || cudaMalloc(&c->d_cent, (size_t)nnz * 8 + 8) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->d_cptr);
    cudaFree(c->d_cent);
    c->d_cptr = nullptr;
    c->d_cent = nullptr;
    return cudaSuccess;
  }
  c->dev_bytes += need + 8;
  if ((e = cudaMemcpyAsync(c->d_cptr, ptr.data(), (rows + 1) * 8, cudaMemcpyHostToDevice, c->st)) != cudaSuccess)
    return e;
  B.count = nullptr;
  B.ptr = c->d_cptr;
  B.ent = c->d_cent;
  if ((e = launch_csr_build(c->G, B, 1, c->span, c->st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(c->st)) != cudaSuccess) return e;
  c->launches++;
  c->csr_nnz = nnz;
  c->csr_state = 1;
  return cudaSuccess;
}

template <int MODE>
static cudaError_t launch_fp(xtg_ctx *c, float *out, double *slots) {
  cudaError_t e = ensure_csr(c);
  if (e != cudaSuccess) return e;
  FpArgs F;
  F.x = c->d_x; F.y = c->d_y; F.d = c->d_d; F.w = c->d_w; F.hr = c->d_hr; F.cosv = c->d_cos; F.sinv = c->d_sin;
  F.fov = c->d_fov; F.out = out; F.cost_slots = slots; F.T = c->g.T; F.delta = c->g.delta;
  F.win_margin = fp_win_margin(c);
  c->launches++;
  if (c->csr_state == 1) {
    CsrView T;
    T.ptr = c->d_cptr;
    T.ent = c->d_cent;
    return xtg::launch_fp_csr(c->G, F, T, MODE, c->st);
  }
  return xtg::launch_fp(c->G, F, MODE, c->span, c->st);
}

extern "C" {

const char *xtg_last_error(void) { return g_err; }
int xtg_abi_version(void) { return XTG_ABI_VERSION; }

void xtg_destroy(xtg_ctx *c) {
  if (!c) return;
  if (c->coarse) xtg_destroy(c->coarse);
  void *ptrs[] = {c->d_y, c->d_w, c->d_e, c->d_d, c->d_x, c->d_mag, c->d_hr, c->d_cos, c->d_sin, c->d_ax,
                  c->d_filt, c->d_tmp, c->d_num, c->d_den, c->d_thr, c->d_var, c->d_view_idx, c->d_view_start,
                  c->d_view_num, c->d_fov, c->d_mcols, c->d_rank, c->d_counter, c->d_nhcnt, c->d_err, c->d_kth,
                  c->d_items, c->d_nh, c->d_red, c->d_absx, c->d_cnt, c->d_tstart, c->d_toff, c->d_tval32,
                  c->d_tscale, c->d_tval16, c->d_rs_hist, c->d_rs_st, c->d_cptr, c->d_cent};
  if (c->dl_pending && c->ev_dl) cudaEventSynchronize(c->ev_dl);
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->d_dl) cudaFree(c->d_dl);
  if (c->ev_dx) cudaEventDestroy(c->ev_dx);
  if (c->ev_dl) cudaEventDestroy(c->ev_dl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ek0) cudaEventDestroy(c->ek0);
  for (cudaEvent_t e : c->tev) cudaEventDestroy(e);
  if (c->ek1) cudaEventDestroy(c->ek1);
  if (c->st) cudaStreamDestroy(c->st);
  if (c->st_copy) cudaStreamDestroy(c->st_copy);
  if (c->ev_y) cudaEventDestroy(c->ev_y);
  if (c->ev_w) cudaEventDestroy(c->ev_w);
  xt_views_free(&c->v);
  delete c;
}

int xtg_create(const xt_params *prm, const double *times, const double *angles, int32_t n, xtg_ctx **out) {
  *out = nullptr;
  if (!prm || !times || !angles || !out) {
    set_err("xtg_create: null argument");
    return XTG_E_ARG;
  }
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0) {
    set_err("xtg_create: no CUDA device (%s); this library has no CPU path", cudaGetErrorString(ce));
    return XTG_E_CUDA;
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) {
    set_err("xtg_create: device %s is sm_%d%d; libxtgpu is built for sm_100a", prop.name, prop.major, prop.minor);
    return XTG_E_CUDA;
  }
  xtg_ctx *c = new xtg_ctx();
  c->prm = *prm;
  c->t_in.assign(times, times + n);
  c->a_in.assign(angles, angles + n);
  char err[512];
  if (xt_geom_derive(prm, &c->g, err, sizeof(err)) != 0) {
    set_err("%s", err);
    delete c;
    return XTG_E_ARG;
  }
  if (xt_views_build(&c->g, times, angles, n, &c->v, err, sizeof(err)) != 0) {
    set_err("%s", err);
    xtg_destroy(c);
    return XTG_E_ARG;
  }
  const xt_geom &g = c->g;
  c->G = make_devgeo(g, prm->positivity);
  c->sm_count = prop.multiProcessorCount;
  c->l2_bytes = prop.l2CacheSize;
  c->ns = (size_t)g.N_p * g.N_r * g.N_t;
  if (c->ns >= ((size_t)1 << 31)) {
    // the kernels address the sinogram with 32-bit entry offsets
    set_err("xtg_create: sinogram of %zu entries exceeds 2^31 - 1", c->ns);
    xtg_destroy(c);
    return XTG_E_ARG;
  }
  c->nrt = (size_t)g.N_r * g.N_t;
  c->nxy = (size_t)g.N_x * g.N_y;
  c->nvox = (size_t)g.N_time * g.N_z * c->nxy;
  c->nmag = (size_t)g.N_time * g.nzb * c->nxy;
  c->hr.resize((size_t)g.N_p * XT_HR_STRIDE);
  xt_detector_response(&g, &c->v, c->hr.data());
  c->col_rank.assign(c->nxy, -1);
  for (int j = 0; j < g.N_y; j++)
    for (int k = 0; k < g.N_x; k++)
      if (xt_in_mask(&g, j, k)) {
        c->col_rank[(size_t)j * g.N_x + k] = (int)c->mcols.size();
        c->mcols.push_back(j * g.N_x + k);
      }
  c->n_masked = (int)c->mcols.size();
  for (int f = 0; f < g.N_time; f++) c->vmax = std::max(c->vmax, c->v.view_num[f]);
  c->span = (int)ceil(2.0 * g.delta_xy / g.delta_r) + 1;  // detector bins a voxel can reach in one view
  rng_seed(c, 761521u);  // the reference seeds once in main (XT_Engine.c:137)

  int rc = 0;
  rc |= dalloc(c, &c->d_y, c->ns);
  rc |= dalloc(c, &c->d_w, c->ns);
  rc |= dalloc(c, &c->d_e, c->ns);
  rc |= dalloc(c, &c->d_d, c->nrt);
  rc |= dalloc(c, &c->d_x, c->nvox);
  rc |= dalloc(c, &c->d_mag, c->nmag);
  rc |= dalloc(c, &c->d_filt, c->nmag);
  rc |= dalloc(c, &c->d_hr, c->hr.size());
  rc |= dalloc(c, &c->d_cos, (size_t)g.N_p);
  rc |= dalloc(c, &c->d_sin, (size_t)g.N_p);
  rc |= dalloc(c, &c->d_num, c->nrt);
  rc |= dalloc(c, &c->d_den, c->nrt);
  rc |= dalloc(c, &c->d_thr, (size_t)g.N_time * g.nzb);
  rc |= dalloc(c, &c->d_kth, (size_t)g.N_time * g.nzb);
  rc |= dalloc(c, &c->d_rs_hist, (size_t)g.N_time * g.nzb * 256);
  rc |= dalloc(c, &c->d_rs_st, (size_t)g.N_time * g.nzb);
  rc |= dalloc(c, &c->d_var, 1);
  rc |= dalloc(c, &c->d_view_idx, (size_t)g.N_p);
  rc |= dalloc(c, &c->d_view_start, (size_t)g.N_time);
  rc |= dalloc(c, &c->d_view_num, (size_t)g.N_time);
  rc |= dalloc(c, &c->d_fov, (size_t)g.N_p);
  rc |= dalloc(c, &c->d_mcols, (size_t)c->n_masked);
  rc |= dalloc(c, &c->d_rank, c->nxy);
  rc |= dalloc(c, &c->d_counter, 8);
  rc |= dalloc(c, &c->d_nhcnt, 2);
  rc |= dalloc(c, &c->d_err, 1);
  rc |= dalloc(c, &c->d_red, 8 * NSLOT);
  rc |= dalloc(c, &c->d_absx, NSLOT);
  rc |= dalloc(c, &c->d_cnt, 4);
  c->items_cap = (size_t)g.N_time * c->n_masked + 1;
  rc |= dalloc(c, &c->d_items, c->items_cap);
  c->nh_cap = (size_t)g.N_time * g.nzb * (c->n_masked / XT_NHICD_CHUNKS + 1) + 2;
  rc |= dalloc(c, &c->d_nh, c->nh_cap);
  if (rc) {
    xtg_destroy(c);
    return XTG_E_CUDA;
  }
  CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  CK(cudaEventCreate(&c->ek0));
  CK(cudaEventCreate(&c->ek1));
  CK(cudaMemcpy(c->d_hr, c->hr.data(), c->hr.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_cos, c->v.cosv, (size_t)g.N_p * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_sin, c->v.sinv, (size_t)g.N_p * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_view_idx, c->v.view_idx, (size_t)g.N_p * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_view_start, c->v.view_start, (size_t)g.N_time * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_view_num, c->v.view_num, (size_t)g.N_time * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_fov, c->v.frame_of_view, (size_t)g.N_p * 4, cudaMemcpyHostToDevice));
  if (c->n_masked) CK(cudaMemcpy(c->d_mcols, c->mcols.data(), (size_t)c->n_masked * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rank, c->col_rank.data(), c->nxy * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_x, 0, c->nvox * 4));
  CK(cudaMemset(c->d_e, 0, c->ns * 4));
  CK(cudaMemset(c->d_d, 0, c->nrt * 4));
  CK(cudaMemset(c->d_mag, 0, c->nmag * 4));
  CK(cudaMemset(c->d_err, 0, 4));
  const float var = g.var_est;
  CK(cudaMemcpy(c->d_var, &var, 4, cudaMemcpyHostToDevice));
  *out = c;
  return XTG_OK;
}

int xtg_dims(const xtg_ctx *c, int32_t *d) {
  if (!c || !d) return XTG_E_ARG;
  const xt_geom &g = c->g;
  d[0] = g.N_x; d[1] = g.N_y; d[2] = g.N_z; d[3] = g.N_time; d[4] = g.N_r; d[5] = g.N_t; d[6] = g.N_p;
  d[7] = g.nzb; d[8] = g.zovl; d[9] = g.amax; d[10] = c->n_masked;
  return 0;
}

int xtg_geometry(const xtg_ctx *c, xt_geom *g) {
  if (!c || !g) return XTG_E_ARG;
  *g = c->g;
  return 0;
}

int xtg_get_hr(const xtg_ctx *c, float *hr) {
  if (!c || !hr) return XTG_E_ARG;
  memcpy(hr, c->hr.data(), c->hr.size() * 4);
  return 0;
}

static int choose_amode(xtg_ctx *c, int *mode);
static int zslab(const xtg_ctx *c);
static int slab_exchange(xtg_ctx *c);

int xtg_set_slab(xtg_ctx *c, float *send_below, float *send_above, const float *recv_below, const float *recv_above,
                 xtg_exchange_fn exchange, void *user) {
  if (!c || (!send_below) != (!recv_below) || (!send_above) != (!recv_above) ||
      ((send_below || send_above) && !exchange)) {
    set_err("xtg_set_slab: each side needs both planes, and planes need an exchange hook");
    return XTG_E_ARG;
  }
  if ((send_below || send_above) && (c->prm.do_VarEst || c->prm.updateProjOffset > 1)) {
    set_err("xtg_set_slab: variance and offset re-estimation need sums over every slab; not supported for slabs");
    return XTG_E_ARG;
  }
  c->send_lo = send_below;
  c->send_hi = send_above;
  c->halo_lo = recv_below;
  c->halo_hi = recv_above;
  c->xfn = (send_below || send_above) ? exchange : nullptr;
  c->xuser = user;
  return 0;
}
int xtg_slab_exchange(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  return slab_exchange(c);
}
int xtg_get_zslab(const xtg_ctx *c, int32_t *slices) {
  if (!c || !slices) return XTG_E_ARG;
  *slices = zslab(c);
  return 0;
}

int xtg_set_zslab(xtg_ctx *c, int32_t slices) {
  if (!c || slices < 0) {
    set_err("xtg_set_zslab: bad argument");
    return XTG_E_ARG;
  }
  c->zslab_req = slices;
  return 0;
}

int xtg_set_options(xtg_ctx *c, int32_t a_mode, int32_t order, int32_t max_columns, uint64_t seed) {
  if (!c || (a_mode != XTG_A_FP32 && a_mode != XTG_A_FP16 && a_mode != XTG_A_TABLE32 && a_mode != XTG_A_AUTO) ||
      (order != XTG_ORDER_PARALLEL && order != XTG_ORDER_SEQUENTIAL) || max_columns < 0) {
    set_err("xtg_set_options: bad option");
    return XTG_E_ARG;
  }
  if (a_mode == XTG_A_AUTO) {
    int rc = choose_amode(c, &a_mode);
    if (rc) return rc;
  }
  if (a_mode != c->a_mode && c->table_mode != 0 && a_mode != XTG_A_FP32) {
    // the entry offsets are shared; only the value array differs between table types
    c->table_mode = 0;
  }
  c->a_mode = a_mode;
  c->order = order;
  c->max_columns = max_columns;
  c->seed = seed;
  return 0;
}

static int check_err_flag(xtg_ctx *c) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->d_err, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (h) {
    CK(cudaMemsetAsync(c->d_err, 0, 4, c->st));
    set_err("non-finite voxel value in an update (theta2 + prior weight <= 0)");
    return XTG_E_NUMERIC;
  }
  return 0;
}

int xtg_upload_sino(xtg_ctx *c, const float *y, const float *w, const float *d) {
  if (!c || !y || !w) {
    set_err("xtg_upload_sino: null argument");
    return XTG_E_ARG;
  }
  CK(cudaMemcpyAsync(c->d_y, y, c->ns * 4, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_w, w, c->ns * 4, cudaMemcpyHostToDevice, c->st));
  if (d)
    CK(cudaMemcpyAsync(c->d_d, d, c->nrt * 4, cudaMemcpyHostToDevice, c->st));
  else
    CK(cudaMemsetAsync(c->d_d, 0, c->nrt * 4, c->st));
  k_scale_weights<<<std::min<unsigned>(blocks_for(c->ns, 256), 4096), 256, 0, c->st>>>(c->ns, c->d_w, c->d_var);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  c->have_sino = 1;
  return 0;
}

// e = y - ax - d from ax already in e, in the order the projector's MODE 1
// applies it (so the result is bit-identical to it)
__global__ void k_e_from_ax(size_t ns, size_t nrt, const float *__restrict__ y, const float *__restrict__ d,
                            float *__restrict__ e) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ns; i += (size_t)gridDim.x * blockDim.x)
    e[i] = __fsub_rn(__fsub_rn(y[i], e[i]), d[i % nrt]);
}

int xtg_upload_sino_start(xtg_ctx *c, const float *y, const float *w, const float *d) {
  if (!c || !y || !w) {
    set_err("xtg_upload_sino_start: null argument");
    return XTG_E_ARG;
  }
  if (!c->st_copy) CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
  if (!c->ev_y) CK(cudaEventCreateWithFlags(&c->ev_y, cudaEventDisableTiming));
  if (!c->ev_w) CK(cudaEventCreateWithFlags(&c->ev_w, cudaEventDisableTiming));
  // Ax of the resident object on the engine's stream (it reads neither y, w
  // nor d) while the measurement crosses on the copy stream
  CK(launch_fp<0>(c, c->d_e, nullptr));
  CK(cudaMemcpyAsync(c->d_y, y, c->ns * 4, cudaMemcpyHostToDevice, c->st_copy));
  if (d)
    CK(cudaMemcpyAsync(c->d_d, d, c->nrt * 4, cudaMemcpyHostToDevice, c->st_copy));
  else
    CK(cudaMemsetAsync(c->d_d, 0, c->nrt * 4, c->st_copy));
  CK(cudaEventRecord(c->ev_y, c->st_copy));
  CK(cudaMemcpyAsync(c->d_w, w, c->ns * 4, cudaMemcpyHostToDevice, c->st_copy));
  CK(cudaEventRecord(c->ev_w, c->st_copy));
  CK(cudaStreamWaitEvent(c->st, c->ev_y, 0));
  k_e_from_ax<<<std::min<unsigned>(blocks_for(c->ns, 256), (unsigned)c->sm_count * 8), 256, 0, c->st>>>(
      c->ns, c->nrt, c->d_y, c->d_d, c->d_e);
  CK(cudaStreamWaitEvent(c->st, c->ev_w, 0));
  k_scale_weights<<<std::min<unsigned>(blocks_for(c->ns, 256), 4096), 256, 0, c->st>>>(c->ns, c->d_w, c->d_var);
  c->launches += 2;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  c->have_sino = 1;
  return 0;
}

int xtg_upload_counts(xtg_ctx *c, const float *bright, const float *counts, double bh, const float *d) {
  if (!c || !bright || !counts) return XTG_E_ARG;
  if (c->prm.sinobin != 3) {
    set_err("xtg_upload_counts: the context was not created with sinobin = 3");
    return XTG_E_STATE;
  }
  const int mxy = (int)c->g.mult_xy, mz = (int)c->g.mult_z;
  const size_t nb = (size_t)c->g.N_r * mxy * c->g.N_t * mz, nc = nb * c->g.N_p;
  float *db = nullptr, *dc = nullptr;
  CK(cudaMalloc(&db, nb * 4));
  if (cudaMalloc(&dc, nc * 4) != cudaSuccess) {
    cudaFree(db);
    set_err("xtg_upload_counts: out of device memory");
    return XTG_E_CUDA;
  }
  cudaMemcpyAsync(db, bright, nb * 4, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(dc, counts, nc * 4, cudaMemcpyHostToDevice, c->st);
  k_counts<<<std::min<unsigned>(blocks_for(c->ns, 256), 8192), 256, 0, c->st>>>(c->G, mxy, mz, db, dc, (float)bh,
                                                                               c->d_y, c->d_w);
  k_scale_weights<<<std::min<unsigned>(blocks_for(c->ns, 256), 4096), 256, 0, c->st>>>(c->ns, c->d_w, c->d_var);
  c->launches += 2;
  if (d)
    cudaMemcpyAsync(c->d_d, d, c->nrt * 4, cudaMemcpyHostToDevice, c->st);
  else
    cudaMemsetAsync(c->d_d, 0, c->nrt * 4, c->st);
  cudaError_t e = cudaStreamSynchronize(c->st);
  cudaFree(db);
  cudaFree(dc);
  CK(e);
  c->have_sino = 1;
  return 0;
}

int xtg_upload_object(xtg_ctx *c, const float *x) {
  if (!c || !x) return XTG_E_ARG;
  if (!c->d_tmp && dalloc(c, &c->d_tmp, c->nvox)) return XTG_E_CUDA;
  CK(cudaMemcpyAsync(c->d_tmp, x, c->nvox * 4, cudaMemcpyHostToDevice, c->st));
  k_obj_h2d<<<std::min<unsigned>(blocks_for(c->nvox, 256), 8192), 256, 0, c->st>>>(c->G, c->d_tmp, c->d_x);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// object from a device buffer in the engine's device layout, 0 outside the
// reconstruction disk and clamped at 0 with positivity
__global__ void k_obj_from_dev(DevGeo G, const int *rank, const float *src, float *dst) {
  const long long n = (long long)G.N_time * G.N_y * G.N_x * G.N_z;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long col = i / G.N_z;
    const int jk = (int)(col % ((long long)G.N_y * G.N_x));
    float v = rank[jk] >= 0 ? src[i] : 0.f;
    if (G.positivity && !(v > 0.f)) v = 0.f;  // also maps NaN to 0
    dst[i] = v;
  }
}

int xtg_object_to_device(xtg_ctx *c, float *dst) {
  if (!c || !dst) return XTG_E_ARG;
  CK(cudaMemcpyAsync(dst, c->d_x, c->nvox * 4, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int xtg_object_from_device(xtg_ctx *c, const float *src) {
  if (!c || !src) return XTG_E_ARG;
  k_obj_from_dev<<<std::min<unsigned>(blocks_for(c->nvox, 256), 8192), 256, 0, c->st>>>(c->G, c->d_rank, src, c->d_x);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// One axis of upsample_object_bilinear_2D/3D (XT_ICD_update.c:354-436): a
// line of n values becomes 2n,
//   out[0] = in[0], out[1] = (3 in[0] + in[1]) / 4,
//   out[2k] = (in[k-1] + 3 in[k]) / 4, out[2k+1] = (3 in[k] + in[k+1]) / 4,
//   out[2n-2] = (in[n-2] + 3 in[n-1]) / 4, out[2n-1] = in[n-1],
// in double and rounded to float once; the reference's y pass writes the
// interior odd rows as (3*b + b') in float first (`3*buffer` is an int times
// a float), reproduced with f32_odd.  Lines are (outer, axis, inner) strided.
__global__ void k_up1d(long long outer, int n, long long inner, const float *in, float *out, int f32_odd) {
  const long long tot = outer * 2 * n * inner;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i % inner;
    const long long q = i / inner;
    const int o = (int)(q % (2 * n));
    const long long b = (q / (2 * n)) * n * inner + r;
    auto at = [&](int k) { return in[b + (long long)k * inner]; };
    float v;
    if (n == 1) {
      v = at(0);
    } else if (o == 0) {
      v = at(0);
    } else if (o == 2 * n - 1) {
      v = at(n - 1);
    } else if (o == 1) {
      v = (float)__dmul_rn(__dadd_rn(__dmul_rn(3.0, (double)at(0)), (double)at(1)), 0.25);
    } else if (o == 2 * n - 2) {
      v = (float)__dmul_rn(__dadd_rn((double)at(n - 2), __dmul_rn(3.0, (double)at(n - 1))), 0.25);
    } else if ((o & 1) == 0) {
      const int k = o / 2;
      v = (float)__dmul_rn(__dadd_rn((double)at(k - 1), __dmul_rn(3.0, (double)at(k))), 0.25);
    } else {
      const int k = o / 2;
      if (f32_odd)
        v = (float)__dmul_rn((double)__fadd_rn(__fmul_rn(3.0f, at(k)), at(k + 1)), 0.25);
      else
        v = (float)__dmul_rn(__dadd_rn(__dmul_rn(3.0, (double)at(k)), (double)at(k + 1)), 0.25);
    }
    out[i] = v;
  }
}

// 2x upsampling of [nt][nz][ny][nx] volumes (in the layout given by the
// strides below) through two scratch buffers: x, then y, then (with_z) z
static int upsample_dev(xtg_ctx *c, const float *in, float *out, int nt, int nz, int ny, int nx, int with_z,
                        bool zfast) {
  const size_t n1 = (size_t)nt * nz * ny * 2 * nx, n2 = n1 * 2;
  float *b1 = nullptr, *b2 = nullptr;
  CK(cudaMalloc(&b1, n1 * 4));
  if (cudaMalloc(&b2, n2 * 4) != cudaSuccess) {
    cudaFree(b1);
    set_err("upsample: out of device memory");
    return XTG_E_CUDA;
  }
  const unsigned g = (unsigned)std::min<size_t>(blocks_for(n2 * 2, 256), (size_t)c->sm_count * 16);
  if (zfast) {  // [t][y][x][z]
    k_up1d<<<g, 256, 0, c->st>>>((long long)nt * ny, nx, nz, in, b1, 0);
    k_up1d<<<g, 256, 0, c->st>>>(nt, ny, (long long)2 * nx * nz, b1, with_z ? b2 : out, 1);
    if (with_z) k_up1d<<<g, 256, 0, c->st>>>((long long)nt * 2 * ny * 2 * nx, nz, 1, b2, out, 0);
  } else {  // [t][z][y][x]
    k_up1d<<<g, 256, 0, c->st>>>((long long)nt * nz * ny, nx, 1, in, b1, 0);
    k_up1d<<<g, 256, 0, c->st>>>((long long)nt * nz, ny, 2 * nx, b1, with_z ? b2 : out, 1);
    if (with_z) k_up1d<<<g, 256, 0, c->st>>>(nt, nz, (long long)4 * ny * nx, b2, out, 0);
  }
  c->launches += with_z ? 3 : 2;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(b1);
  cudaFree(b2);
  if (e != cudaSuccess) {
    set_err("upsample: %s", cudaGetErrorString(e));
    return XTG_E_CUDA;
  }
  return 0;
}

int xtg_upsample(xtg_ctx *c, const float *in, float *out, int32_t nt, int32_t nz, int32_t ny, int32_t nx,
                 int32_t with_z) {
  if (!c || !in || !out || nt < 1 || nz < 1 || ny < 1 || nx < 1) return XTG_E_ARG;
  const size_t nin = (size_t)nt * nz * ny * nx, nout = nin * (with_z ? 8 : 4);
  float *din = nullptr, *dout = nullptr;
  CK(cudaMalloc(&din, nin * 4));
  if (cudaMalloc(&dout, nout * 4) != cudaSuccess) {
    cudaFree(din);
    set_err("xtg_upsample: out of device memory");
    return XTG_E_CUDA;
  }
  int rc = 0;
  if (cudaMemcpy(din, in, nin * 4, cudaMemcpyHostToDevice) != cudaSuccess) rc = XTG_E_CUDA;
  if (!rc) rc = upsample_dev(c, din, dout, nt, nz, ny, nx, with_z, false);
  if (!rc && cudaMemcpy(out, dout, nout * 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = XTG_E_CUDA;
  cudaFree(din);
  cudaFree(dout);
  return rc;
}

// 2 x 2 (or 2 x 1) detector binning for the binned coarse problem: weights
// add (as counts do, genSinogram_subsampleCounts, XT_genSinogram.c:303-374, sums them),
// the projection is the weight-averaged one, the offset the plain mean
__global__ void k_bin_sino(int np, int nrc, int ntc, int nrf, int ntf, int fr, int ft, const float *y, const float *w,
                           const float *d, float *yc, float *wc, float *dc) {
  const long long n = (long long)np * nrc * ntc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i % ntc);
    const long long q = i / ntc;
    const int r = (int)(q % nrc), p = (int)(q / nrc);
    double W = 0, WY = 0, Y = 0, D = 0;
    for (int a = 0; a < fr; a++)
      for (int b = 0; b < ft; b++) {
        const size_t f = ((size_t)p * nrf + r * fr + a) * ntf + t * ft + b;
        W += w[f];
        WY += (double)w[f] * y[f];
        Y += y[f];
        if (p == 0) D += d[(size_t)(r * fr + a) * ntf + t * ft + b];
      }
    wc[i] = (float)W;
    yc[i] = (float)(W > 0 ? WY / W : Y / (fr * ft));
    if (p == 0) dc[(size_t)r * ntc + t] = (float)(D / (fr * ft));
  }
}

extern "C" int xtg_init_error_model(xtg_ctx *c);

int xtg_init_object_multires(xtg_ctx *c, int32_t coarse_iters, int32_t flags) {
  if (!c || coarse_iters < 0 || (flags & ~(XTG_MULTIRES_Z | XTG_MULTIRES_BIN))) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_init_object_multires: no sinogram uploaded");
    return XTG_E_STATE;
  }
  const xt_geom &g = c->g;
  // a counts-ingested sinogram (sinobin 3) is already binned to the voxel
  // size, so its coarse stage bins it further, as the reference's counts
  // ingest does at each stage of the launcher
  if (c->prm.sinobin == 3) flags |= XTG_MULTIRES_BIN;
  const bool with_z = flags & XTG_MULTIRES_Z, bin = flags & XTG_MULTIRES_BIN;
  if (g.N_x % 2 || g.N_y % 2 || (with_z && g.N_z % 2)) {
    set_err("xtg_init_object_multires: grid not divisible by 2");
    return XTG_E_ARG;
  }
  if (c->coarse && c->coarse_flags != flags) {
    xtg_destroy(c->coarse);
    c->coarse = nullptr;
  }
  if (!c->coarse) {
    // the same scan with voxels twice as large (the launcher's coarser
    // stage); binned, its detector bins (and rows) are twice as large too,
    // the geometry counts ingest derives (sinobin 3: N_r / delta_xy bins of
    // delta_xy fine bins, priors scaled by delta_xy as on the unbinned grid)
    xt_params cp = c->prm;
    cp.delta_xy *= 2;
    if (with_z) cp.delta_z *= 2;
    if (bin) cp.sinobin = 3;
    int rc = xtg_create(&cp, c->t_in.data(), c->a_in.data(), (int32_t)c->t_in.size(), &c->coarse);
    if (rc) return rc;
    c->coarse_flags = flags;
    if ((rc = xtg_set_options(c->coarse, c->a_mode, XTG_ORDER_PARALLEL, c->max_columns, c->seed))) return rc;
  }
  xtg_ctx *cc = c->coarse;
  // fine detector bins (rows) per coarse one: 2 binned from voxel-sized bins,
  // 2 delta_xy (2 delta_z) from bins of a grid with delta_xy > 1
  const int fr = g.N_r / cc->g.N_r, ft = g.N_t / cc->g.N_t;
  if (cc->g.N_x * 2 != g.N_x || cc->g.N_y * 2 != g.N_y || cc->g.N_z * (with_z ? 2 : 1) != g.N_z ||
      cc->g.N_p != g.N_p || cc->g.N_r * fr != g.N_r || cc->g.N_t * ft != g.N_t || (!bin && (fr != 1 || ft != 1))) {
    set_err("xtg_init_object_multires: the coarse grid is not half the fine one");
    return XTG_E_ARG;
  }
  if (bin) {
    // the binned measurement; weights are already scaled by the variance
    const unsigned gr = (unsigned)std::min<size_t>((cc->ns + 255) / 256, (size_t)c->sm_count * 16);
    k_bin_sino<<<gr, 256, 0, c->st>>>(g.N_p, cc->g.N_r, cc->g.N_t, g.N_r, g.N_t, fr, ft, c->d_y, c->d_w, c->d_d,
                                      cc->d_y, cc->d_w, cc->d_d);
    c->launches++;
    CK(cudaGetLastError());
  } else {
    // the same measurement, weights (already scaled by the variance) and offset
    CK(cudaMemcpyAsync(cc->d_y, c->d_y, c->ns * 4, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(cc->d_w, c->d_w, c->ns * 4, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(cc->d_d, c->d_d, c->nrt * 4, cudaMemcpyDeviceToDevice, c->st));
  }
  CK(cudaMemcpyAsync(cc->d_var, c->d_var, 4, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  cc->have_sino = 1;
  int rc = xtg_init_object_fbp(cc);
  for (int it = 1; it <= coarse_iters && !rc; it++) rc = xtg_icd_iteration(cc, it, nullptr);
  if (rc) return rc;
  const xt_geom &h = cc->g;
  if (!c->d_tmp && dalloc(c, &c->d_tmp, c->nvox)) return XTG_E_CUDA;
  rc = upsample_dev(c, cc->d_x, c->d_tmp, h.N_time, h.N_z, h.N_y, h.N_x, with_z, true);
  if (rc) return rc;
  rc = xtg_object_from_device(c, c->d_tmp);
  if (rc) return rc;
  return xtg_init_error_model(c);
}

int xtg_download_object(xtg_ctx *c, float *x) {
  if (!c || !x) return XTG_E_ARG;
  if (!c->d_tmp && dalloc(c, &c->d_tmp, c->nvox)) return XTG_E_CUDA;
  k_obj_d2h<<<std::min<unsigned>(blocks_for(c->nvox, 256), 8192), 256, 0, c->st>>>(c->G, c->d_x, c->d_tmp);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(x, c->d_tmp, c->nvox * 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// The object leaves for the host without blocking it: transposed into its own
// staging buffer on the engine's stream (later kernels may change x at once),
// then copied on the copy stream, so the copy overlaps whatever the host
// queues next (the next sinogram's upload and projection).  A second call
// first waits for the previous copy to leave the staging buffer.
int xtg_download_object_start(xtg_ctx *c, float *x) {
  if (!c || !x) return XTG_E_ARG;
  if (!c->st_copy) CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
  if (!c->ev_dx) CK(cudaEventCreateWithFlags(&c->ev_dx, cudaEventDisableTiming));
  if (!c->ev_dl) CK(cudaEventCreateWithFlags(&c->ev_dl, cudaEventDisableTiming));
  if (!c->d_dl && dalloc(c, &c->d_dl, c->nvox)) return XTG_E_CUDA;
  if (c->dl_pending) CK(cudaStreamWaitEvent(c->st, c->ev_dl, 0));
  k_obj_d2h<<<std::min<unsigned>(blocks_for(c->nvox, 256), 8192), 256, 0, c->st>>>(c->G, c->d_x, c->d_dl);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev_dx, c->st));
  CK(cudaStreamWaitEvent(c->st_copy, c->ev_dx, 0));
  CK(cudaMemcpyAsync(x, c->d_dl, c->nvox * 4, cudaMemcpyDeviceToHost, c->st_copy));
  CK(cudaEventRecord(c->ev_dl, c->st_copy));
  c->dl_pending = 1;
  return 0;
}

int xtg_download_wait(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  if (c->dl_pending) {
    CK(cudaEventSynchronize(c->ev_dl));
    c->dl_pending = 0;
  }
  return 0;
}

#define XTG_COPY_FN(name, dev, count, kind, ptype)                        \
  int name(xtg_ctx *c, ptype p) {                                         \
    if (!c || !p) return XTG_E_ARG;                                       \
    CK(cudaMemcpyAsync((void *)(kind == cudaMemcpyDeviceToHost ? (void *)p : (void *)c->dev), \
                       (const void *)(kind == cudaMemcpyDeviceToHost ? (const void *)c->dev : (const void *)p), \
                       (count) * 4, kind, c->st));                        \
    CK(cudaStreamSynchronize(c->st));                                     \
    return 0;                                                             \
  }
XTG_COPY_FN(xtg_get_error_sino, d_e, c->ns, cudaMemcpyDeviceToHost, float *)
XTG_COPY_FN(xtg_set_error_sino, d_e, c->ns, cudaMemcpyHostToDevice, const float *)
XTG_COPY_FN(xtg_get_weight, d_w, c->ns, cudaMemcpyDeviceToHost, float *)
XTG_COPY_FN(xtg_get_offset, d_d, c->nrt, cudaMemcpyDeviceToHost, float *)
XTG_COPY_FN(xtg_set_offset, d_d, c->nrt, cudaMemcpyHostToDevice, const float *)
XTG_COPY_FN(xtg_get_magmap, d_mag, c->nmag, cudaMemcpyDeviceToHost, float *)
XTG_COPY_FN(xtg_set_magmap, d_mag, c->nmag, cudaMemcpyHostToDevice, const float *)

int xtg_get_variance(xtg_ctx *c, double *v) {
  if (!c || !v) return XTG_E_ARG;
  float h = 0;
  CK(cudaMemcpyAsync(&h, c->d_var, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *v = h;
  return 0;
}

int xtg_set_variance(xtg_ctx *c, double v) {
  if (!c || !(v > 0)) return XTG_E_ARG;
  const float h = (float)v;
  CK(cudaMemcpyAsync(c->d_var, &h, 4, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int xtg_amatrix(xtg_ctx *c, int32_t n, const int32_t *rows, const int32_t *cols, const int32_t *views, float *vals,
                int32_t *idx, int32_t *cnt) {
  if (!c || n < 0 || (n && (!rows || !cols || !views || !vals || !idx || !cnt))) return XTG_E_ARG;
  if (n == 0) return 0;
  for (int i = 0; i < n; i++)
    if (rows[i] < 0 || rows[i] >= c->g.N_y || cols[i] < 0 || cols[i] >= c->g.N_x || views[i] < 0 ||
        views[i] >= c->g.N_p) {
      set_err("xtg_amatrix: triple %d out of range", i);
      return XTG_E_ARG;
    }
  int *dr, *dcol, *dv, *di, *dc;
  float *dval;
  const size_t na = (size_t)n * c->g.amax;
  CK(cudaMalloc(&dr, (size_t)n * 4 * 3 + (size_t)n * 4 + na * 8));
  dcol = dr + n;
  dv = dcol + n;
  dc = dv + n;
  dval = reinterpret_cast<float *>(dc + n);
  di = reinterpret_cast<int *>(dval + na);
  cudaMemcpyAsync(dr, rows, (size_t)n * 4, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(dcol, cols, (size_t)n * 4, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(dv, views, (size_t)n * 4, cudaMemcpyHostToDevice, c->st);
  k_amatrix_batch<<<blocks_for(n, 128), 128, 0, c->st>>>(c->G, c->d_hr, c->d_cos, c->d_sin, n, dr, dcol, dv, dval, di, dc);
  c->launches++;
  cudaMemcpyAsync(vals, dval, na * 4, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(idx, di, na * 4, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(cnt, dc, (size_t)n * 4, cudaMemcpyDeviceToHost, c->st);
  cudaError_t e = cudaStreamSynchronize(c->st);
  cudaFree(dr);
  CK(e);
  return 0;
}

int xtg_forward_project(xtg_ctx *c, float *ax) {
  if (!c) return XTG_E_ARG;
  if (!c->d_ax && dalloc(c, &c->d_ax, c->ns)) return XTG_E_CUDA;
  CK(launch_fp<0>(c, c->d_ax, nullptr));
  if (ax) CK(cudaMemcpyAsync(ax, c->d_ax, c->ns * 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int xtg_init_error_sino(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_init_error_sino: no sinogram uploaded");
    return XTG_E_STATE;
  }
  CK(launch_fp<1>(c, c->d_e, nullptr));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int finish_cost(xtg_ctx *c, double data_sum, double *cost, double *fwd, double *prior);

// e for a start this library computed itself (FBP, multi-resolution, the
// network): e = y - A delta_t x - d, the error sinogram of the matrix the
// voxel update uses, so ICD continues from a consistent state.  With
// delta_t = 1 that is the reference's projection (bit-exact FP32 path);
// otherwise the FP64 pass rounded to FP32 (the reference's own projector
// leaves out delta_t, which only its zero start makes harmless).
__attribute__((visibility("hidden"))) int xtg_init_error_model(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  if (c->g.delta_t == 1.0f) return xtg_init_error_sino(c);
  return xtg_resync_fp64(c, nullptr, nullptr, nullptr);
}

// the FBP image into the object, leaving e stale (filtered sinogram in it):
// for callers inside the library that replace the object again before they
// iterate (not exported)
__attribute__((visibility("hidden"))) int xtg_fbp_image_only(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_init_object_fbp: no sinogram uploaded");
    return XTG_E_STATE;
  }
  // the filtered sinogram lives in e until e = y - Ax - d overwrites it
  CK(launch_fbp(c->G, c->d_y, c->d_d, c->d_e, c->d_cos, c->d_sin, c->d_view_idx, c->d_view_start, c->d_view_num,
                c->d_rank, c->d_x, c->st));
  c->launches += 2;
  return 0;
}

int xtg_init_object_fbp(xtg_ctx *c) {
  const int rc = xtg_fbp_image_only(c);
  return rc ? rc : xtg_init_error_model(c);
}

int xtg_resync_fp64(xtg_ctx *c, double *cost, double *fwd, double *prior) {
  if (!c) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_resync_fp64: no sinogram uploaded");
    return XTG_E_STATE;
  }
  CK(cudaMemsetAsync(c->d_red, 0, NSLOT * 8, c->st));
  CK(launch_fp<2>(c, c->d_e, c->d_red));
  if (!cost && !fwd && !prior) {
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  double h[NSLOT];
  CK(cudaMemcpyAsync(h, c->d_red, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double s = 0;
  for (int i = 0; i < NSLOT; i++) s += h[i];
  return finish_cost(c, s, cost, fwd, prior);
}

static int finish_cost(xtg_ctx *c, double data_sum, double *cost, double *fwd, double *prior) {
  CK(cudaMemsetAsync(c->d_red + NSLOT, 0, NSLOT * 8, c->st));
  // one warp per z-line, 8 warps per CTA
  const unsigned grid = std::min<unsigned>(blocks_for((size_t)c->g.N_time * c->g.N_y * c->g.N_x, 8),
                                           (unsigned)c->sm_count * 8);
  k_prior_cost64<<<grid, 256, 0, c->st>>>(c->G, c->d_x, c->halo_hi, c->d_red + NSLOT);
  c->launches++;
  CK(cudaGetLastError());
  double h[NSLOT];
  CK(cudaMemcpyAsync(h, c->d_red + NSLOT, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  float var = 0;
  CK(cudaMemcpyAsync(&var, c->d_var, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double pr = 0;
  for (int i = 0; i < NSLOT; i++) pr += h[i];
  const double f = data_sum / 2.0 + (double)c->g.N_p * c->g.N_r * c->g.N_t * log((double)var) / 2.0;
  if (cost) *cost = f + pr;
  if (fwd) *fwd = f;
  if (prior) *prior = pr;
  return 0;
}

int xtg_map_cost_fp64(xtg_ctx *c, double *cost, double *fwd, double *prior) {
  if (!c) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_map_cost_fp64: no sinogram uploaded");
    return XTG_E_STATE;
  }
  CK(cudaMemsetAsync(c->d_red, 0, NSLOT * 8, c->st));
  CK(launch_fp<3>(c, nullptr, c->d_red));
  double h[NSLOT];
  CK(cudaMemcpyAsync(h, c->d_red, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double s = 0;
  for (int i = 0; i < NSLOT; i++) s += h[i];
  return finish_cost(c, s, cost, fwd, prior);
}

int xtg_map_cost_running(xtg_ctx *c, double *cost, double *fwd, double *prior) {
  if (!c) return XTG_E_ARG;
  CK(cudaMemsetAsync(c->d_red, 0, NSLOT * 8, c->st));
  const unsigned grid = std::min<unsigned>(blocks_for(c->ns, 256), (unsigned)c->sm_count * 8);
  k_running_cost64<<<grid, 256, 0, c->st>>>(c->ns, c->d_e, c->d_w, c->g.T, c->g.delta, c->d_red);
  c->launches++;
  CK(cudaGetLastError());
  double h[NSLOT];
  CK(cudaMemcpyAsync(h, c->d_red, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double s = 0;
  for (int i = 0; i < NSLOT; i++) s += h[i];
  return finish_cost(c, s, cost, fwd, prior);
}

int xtg_zinger_refresh(xtg_ctx *c, uint8_t *sel, int64_t *nsel) {
  if (!c) return XTG_E_ARG;
  unsigned char *ds = nullptr;
  if (sel) CK(cudaMalloc(&ds, c->ns));
  CK(cudaMemsetAsync(c->d_cnt + 3, 0, 8, c->st));
  const unsigned grid = std::min<unsigned>(blocks_for(c->ns, 256), (unsigned)c->sm_count * 8);
  k_zinger_refresh<<<grid, 256, 0, c->st>>>(c->ns, c->d_e, c->d_w, c->g.T, ds, c->d_cnt + 3);
  c->launches++;
  unsigned long long h = 0;
  cudaMemcpyAsync(&h, c->d_cnt + 3, 8, cudaMemcpyDeviceToHost, c->st);
  if (sel) cudaMemcpyAsync(sel, ds, c->ns, cudaMemcpyDeviceToHost, c->st);
  cudaError_t e = cudaStreamSynchronize(c->st);
  if (ds) cudaFree(ds);
  CK(e);
  if (nsel) *nsel = (int64_t)h;
  return 0;
}

int xtg_update_offset(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  CK(cudaMemsetAsync(c->d_red + 2 * NSLOT, 0, 2 * 8, c->st));
  const unsigned grid = blocks_for(c->nrt, 128);
  k_offset_numden<<<grid, 128, 0, c->st>>>(c->G, c->d_e, c->d_w, c->d_d, c->d_num, c->d_den, c->d_red + 2 * NSLOT);
  k_offset_apply<<<grid, 128, 0, c->st>>>(c->G, c->d_e, c->d_d, c->d_num, c->d_den, c->d_red + 2 * NSLOT,
                                          c->prm.EnforceZeroMeanOffset);
  c->launches += 2;
  CK(cudaGetLastError());
  return 0;
}

int xtg_update_variance(xtg_ctx *c) {
  if (!c) return XTG_E_ARG;
  CK(cudaMemsetAsync(c->d_red + 3 * NSLOT, 0, NSLOT * 8, c->st));
  const unsigned grid = std::min<unsigned>(blocks_for(c->ns, 256), (unsigned)c->sm_count * 8);
  k_var_sum<<<grid, 256, 0, c->st>>>(c->ns, c->d_e, c->d_w, c->d_var, c->g.T, c->g.delta, c->d_red + 3 * NSLOT);
  k_var_finish<<<1, 32, 0, c->st>>>(c->d_red + 3 * NSLOT, (double)c->ns, c->d_var);
  k_scale_weights<<<grid, 256, 0, c->st>>>(c->ns, c->d_w, c->d_var);
  c->launches += 3;
  CK(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------ ICD driver --
// Builds the A-matrix column table for the current a_mode (count pass, host
// prefix sum, fill pass).  Rebuilt only when the value type changes.
static TableArgs table_args(const xtg_ctx *c) {
  TableArgs T;
  memset(&T, 0, sizeof(T));
  T.hr = c->d_hr; T.cosv = c->d_cos; T.sinv = c->d_sin; T.view_idx = c->d_view_idx; T.view_start = c->d_view_start;
  T.view_num = c->d_view_num; T.mcols = c->d_mcols; T.n_masked = c->n_masked;
  return T;
}

// Entries per (frame, masked column) over the frame's views, turned into run
// starts on the host; returns the total and the longest run.
static int count_table(xtg_ctx *c, std::vector<long long> &cnt, long long *total, long long *longest) {
  const size_t ncol = (size_t)c->g.N_time * c->n_masked;
  TableArgs T = table_args(c);
  if (!c->d_tstart && dalloc(c, &c->d_tstart, ncol + 1)) return XTG_E_CUDA;
  CK(launch_table_count(c->G, T, c->span, c->d_tstart, c->st));
  c->launches++;
  cnt.assign(ncol + 1, 0);
  CK(cudaMemcpyAsync(cnt.data(), c->d_tstart, ncol * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  long long run = 0, mx = 0;
  for (size_t i = 0; i < ncol; i++) {
    const long long n = cnt[i];
    cnt[i] = run;
    run += n;
    mx = std::max(mx, n);
  }
  cnt[ncol] = run;
  *total = run;
  *longest = mx;
  return 0;
}

// XTG_A_AUTO: the exact FP32 table when it fits in free device memory with
// 2 GiB to spare, else the FP16 table, else entries computed per visit.
int xtg_set_projector(xtg_ctx *c, int32_t kind) {
  if (!c || (kind != XTG_PROJ_AUTO && kind != XTG_PROJ_GATHER)) {
    set_err("xtg_set_projector: bad projector kind");
    return XTG_E_ARG;
  }
  if (kind != c->projector) {
    cudaFree(c->d_cptr);
    cudaFree(c->d_cent);
    if (c->csr_state == 1) c->dev_bytes -= (size_t)c->csr_nnz * 8 + ((size_t)c->g.N_p * c->g.N_r + 2) * 8;
    c->d_cptr = nullptr;
    c->d_cent = nullptr;
    c->csr_state = 0;
    c->csr_nnz = 0;
    c->projector = kind;
  }
  return 0;
}
int xtg_get_projector(const xtg_ctx *c, int32_t *in_use, int64_t *table_entries) {
  if (!c) return XTG_E_ARG;
  if (in_use) *in_use = c->csr_state == 1 ? XTG_PROJ_TABLE : c->csr_state == -1 ? XTG_PROJ_GATHER : XTG_PROJ_AUTO;
  if (table_entries) *table_entries = c->csr_nnz;
  return 0;
}
int xtg_get_options(const xtg_ctx *c, int32_t *a_mode, int32_t *order, int32_t *max_columns, uint64_t *seed) {
  if (!c) return XTG_E_ARG;
  if (a_mode) *a_mode = c->a_mode;
  if (order) *order = c->order;
  if (max_columns) *max_columns = c->max_columns;
  if (seed) *seed = c->seed;
  return 0;
}
static int choose_amode(xtg_ctx *c, int *mode) {
  std::vector<long long> cnt;
  long long run = 0, mx = 0;
  int rc = count_table(c, cnt, &run, &mx);
  if (rc) return rc;
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  const size_t reserve = (size_t)2 << 30, ncol = (size_t)c->g.N_time * c->n_masked;
  if ((size_t)run * 8 + reserve < fr)
    *mode = XTG_A_TABLE32;
  else if ((size_t)run * 6 + ncol * 4 + reserve < fr)
    *mode = XTG_A_FP16;
  else
    *mode = XTG_A_FP32;
  return 0;
}

static int ensure_table(xtg_ctx *c) {
  if (c->table_mode == c->a_mode) return 0;
  const size_t ncol = (size_t)c->g.N_time * c->n_masked;
  TableArgs T = table_args(c);
  std::vector<long long> cnt;
  long long run = 0, mx = 0;
  int rc = count_table(c, cnt, &run, &mx);
  if (rc) return rc;
  if (c->d_toff && c->table_nnz != run) {
    set_err("A table size changed");
    return XTG_E_STATE;
  }
  c->table_nnz = run;
  c->table_max = (int)mx;
  CK(cudaMemcpyAsync(c->d_tstart, cnt.data(), (ncol + 1) * 8, cudaMemcpyHostToDevice, c->st));
  if (!c->d_toff && dalloc(c, &c->d_toff, (size_t)run)) return XTG_E_CUDA;
  if (c->a_mode == XTG_A_FP16) {
    if (!c->d_tval16 && dalloc(c, &c->d_tval16, (size_t)run)) return XTG_E_CUDA;
    if (!c->d_tscale && dalloc(c, &c->d_tscale, ncol)) return XTG_E_CUDA;
    T.val16 = c->d_tval16;
    T.scale = c->d_tscale;
  } else {
    if (!c->d_tval32 && dalloc(c, &c->d_tval32, (size_t)run)) return XTG_E_CUDA;
    T.val32 = c->d_tval32;
  }
  T.start = c->d_tstart;
  T.off = c->d_toff;
  CK(launch_table_fill(c->G, T, c->span, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->launches++;
  c->table_mode = c->a_mode;
  return 0;
}

// z slices per ICD work piece.  Whole z-lines by default: every piece
// restages the column's A entries, so on the plain-3D-at-scale workload
// (512^2 x 64) pieces sized to keep the e and w rows in flight inside L2
// (16 slices) ran 19 % slower than whole lines.  Lines longer than the
// kernel's row limit (128 detector rows with 16-byte access, else 32) are cut
// into equal pieces whose rows keep 16-byte alignment.
static int zslab(const xtg_ctx *c) {
  const xt_geom &g = c->g;
  if (c->zslab_req > 0) return std::min(c->zslab_req, g.N_z);
  const int max_rows = (g.N_t % 4 == 0) ? 128 : 32;
  const int fit = std::max(1, max_rows / g.zovl);
  if (g.N_z <= fit) return g.N_z;
  const int npiece = (g.N_z + fit - 1) / fit;
  int hz = (g.N_z + npiece - 1) / npiece;
  if (g.N_t % 4 == 0) {
    const int q = 4 / std::gcd(4, g.zovl);  // slices per 4 rows
    hz = (hz + q - 1) / q * q;
    if (hz > fit) hz = fit / q * q;
  }
  return std::max(1, hz);
}

// one ICD launch over items[lo, lo+n) (or a device-counted list)
static int run_columns(xtg_ctx *c, int iter, const int4 *items, int lo, int n, const int *n_dev, int use_perm,
                       unsigned long long key, int has_whole, int has_blocks, int seq_override) {
  const xt_geom &g = c->g;
  if (c->a_mode != XTG_A_FP32) {
    int rc = ensure_table(c);
    if (rc) return rc;
  }
  const int seq = (seq_override >= 0) ? seq_override : (c->order == XTG_ORDER_SEQUENTIAL);
  // slices of the largest work item: a whole z-line, or one z-block (the
  // last block is the longest)
  const int last_block = g.N_z - (g.nzb - 1) * g.zstep;
  const int zitem = has_whole ? g.N_z : last_block;
  // the parallel schedule splits items into z pieces of at most hz slices
  // and visits them piece-major; shared memory is sized for one piece
  const int hz = seq ? zitem : std::min(zitem, zslab(c));
  const int nsub = (zitem + hz - 1) / hz;
  const int zmax = hz;
  const int rows = zmax * g.zovl;
  // 16-byte vector access needs every piece's first row and row count to be
  // multiples of 4
  bool v4 = (g.N_t % 4 == 0);
  auto pieces_ok = [&](int z0, int len) {
    for (int o = 0; o < len; o += hz) {
      const int l = std::min(hz, len - o);
      if (((z0 + o) * g.zovl) % 4 || (l * g.zovl) % 4) return false;
    }
    return true;
  };
  if (has_whole) v4 = v4 && pieces_ok(0, g.N_z);
  if (has_blocks)
    for (int b = 0; b < g.nzb && v4; b++) v4 = pieces_ok(b * g.zstep, b == g.nzb - 1 ? last_block : g.zstep);
  const int vec = v4 ? 4 : 1;
  if ((rows + vec - 1) / vec > 32) {
    set_err("ICD work item of %d detector rows exceeds the kernel's %d (N_z/nzb too large)", rows, 32 * vec);
    return XTG_E_ARG;
  }
  const int span = c->span;
  const int as = span <= 3 ? 3 : span <= 4 ? 4 : 12;
  if (span > 12) {
    set_err("delta_xy too large for the ICD kernel (%d bins per view)", span);
    return XTG_E_ARG;
  }
  const int amode = (c->a_mode == XTG_A_FP16) ? 1 : (c->a_mode == XTG_A_TABLE32) ? 2 : 0;
  // shared memory per CTA: per-view slots (A in the kernel) or the longest column run (table)
  const int vcap = amode ? c->table_max : c->vmax;
  IcdArgs A;
  memset(&A, 0, sizeof(A));
  A.e = c->d_e; A.w = c->d_w; A.x = c->d_x; A.magmap = c->d_mag; A.hr = c->d_hr; A.cosv = c->d_cos;
  A.sinv = c->d_sin; A.view_idx = c->d_view_idx; A.view_start = c->d_view_start; A.view_num = c->d_view_num;
  A.items = items; A.n_items_dev = n_dev; A.n_items = n; A.item_lo = lo; A.counter = c->d_counter;
  A.use_perm = use_perm; A.perm_key = key; A.col_rank = c->d_rank; A.n_masked = c->n_masked; A.iter = iter;
  A.tstart = c->d_tstart; A.toff = c->d_toff; A.tval32 = c->d_tval32; A.tval16 = c->d_tval16; A.tscale = c->d_tscale;
  A.T2 = g.T * g.T; A.Tdelta = g.T * g.delta; A.st_absx = c->d_absx; A.st_cnt = c->d_cnt; A.err = c->d_err;
  A.zslab = hz; A.nsub = nsub;
  A.halo_lo = c->halo_lo; A.halo_hi = c->halo_hi;
  A.w_keep = XTG_W_KEEP && 2 * c->ns * 4 <= (size_t)XTG_W_KEEP_BYTES;
  if (nsub > 1) {
    CK(launch_magmap_zero(c->G, A, c->sm_count * 4, c->st));
    c->launches++;
  }
  int grid;
  if (seq) {
    grid = 1;
  } else {
    const int occ = icd_occupancy(vec, amode, 0, as, vcap, zmax, g.zovl);
    grid = c->sm_count * occ;
    // Columns updated at the same time read each other's stale error
    // sinogram; near neighbours share most of their footprint, so too many
    // of them at once overshoot (Jacobi-like) and the cost stops falling.
    // At most 1 in XTG_CONC_DIV of the grid's columns is in flight: on a
    // 32^2-column grid 64 and more at once left the cost oscillating 20-50 %
    // above the converged value, 32 did not; grids of 256^2 columns and up
    // keep every resident CTA busy.
    grid = std::min(grid, std::max(8, (int)(((long long)g.N_time * c->n_masked) / XTG_CONC_DIV)));
    if (c->max_columns > 0) grid = std::min(grid, c->max_columns);
    if (!n_dev) grid = std::min(grid, std::max(n * nsub, 1));
  }
  CK(cudaMemsetAsync(c->d_counter, 0, 4, c->st));
  CK(launch_icd(c->G, A, vec, amode, seq, as, vcap, zmax, grid, c->st));
  c->icd_launches++;
  c->launches++;
  return 0;
}

static void magsum_launch(xtg_ctx *c) {
  const size_t n = (size_t)c->g.N_time * c->g.nzb * c->n_masked;
  const unsigned grid = std::min<unsigned>(blocks_for(n, 256), (unsigned)c->sm_count * 4);
  k_magsum<<<std::max(grid, 1u), 256, 0, c->st>>>(c->G, c->n_masked, c->d_mcols, c->d_mag, c->d_red + 4 * NSLOT);
  c->launches++;
}

// k-th smallest of each of nseg segments of c->d_filt (k from c->d_kth) into
// c->d_thr: four 8-bit passes, each a histogram over many CTAs and a pick
static void radix_select_multi(xtg_ctx *c, int nseg) {
  const int seglen = (int)c->nxy;
  const int parts = std::max(1, std::min(64, (seglen + 8191) / 8192));
  k_rs_init<<<nseg, 256, 0, c->st>>>(c->d_kth, c->d_rs_st, c->d_rs_hist);
  for (int shift = 24; shift >= 0; shift -= 8) {
    k_rs_hist<<<dim3((unsigned)parts, (unsigned)nseg), 256, 0, c->st>>>(c->d_filt, seglen, shift, c->d_rs_st,
                                                                       c->d_rs_hist);
    k_rs_pick<<<nseg, 256, 0, c->st>>>(shift, c->d_rs_st, c->d_rs_hist, c->d_thr);
  }
  c->launches += 9;
}

// NHICD selection on the device: filter, per-(frame, block) order statistic,
// compaction into the two half-pass lists.
static int nhicd_select_device(xtg_ctx *c) {
  const xt_geom &g = c->g;
  const int nseg = g.N_time * g.nzb;
  const int nsel = c->n_masked / XT_NHICD_CHUNKS;
  std::vector<int> kth(nseg, (int)c->nxy - nsel);
  CK(cudaMemcpyAsync(c->d_kth, kth.data(), nseg * 4, cudaMemcpyHostToDevice, c->st));
  const unsigned grid = std::min<unsigned>(blocks_for(c->nmag, 256), (unsigned)c->sm_count * 8);
  k_vsc_filter<<<grid, 256, 0, c->st>>>(nseg, g.N_y, g.N_x, c->d_mag, c->d_filt);
  radix_select_multi(c, nseg);
  CK(cudaMemsetAsync(c->d_nhcnt, 0, 8, c->st));
  const int cap0 = (int)(c->nh_cap / 2), cap1 = (int)(c->nh_cap - c->nh_cap / 2);
  k_nhicd_compact<<<grid, 256, 0, c->st>>>(g.N_time, g.nzb, g.N_y, g.N_x, c->d_filt, c->d_thr, c->d_rank,
                                           c->d_mag, c->d_nh, c->d_nh + cap0, c->d_nhcnt, cap0, cap1);
  k_clamp_count<<<1, 32, 0, c->st>>>(c->d_nhcnt, cap0, cap1);
  c->launches += 3;
  CK(cudaGetLastError());
  return 0;
}

static int read_stats(xtg_ctx *c, xtg_stats *st, double *absx_out) {
  double ab[NSLOT];
  unsigned long long cnt[3];
  CK(cudaMemcpyAsync(ab, c->d_absx, sizeof(ab), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(cnt, c->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double s = 0;
  for (int i = 0; i < NSLOT; i++) s += ab[i];
  if (absx_out) *absx_out = s;
  if (st) {
    st->voxel_updates += (int64_t)cnt[0];
    st->zero_skipped += (int64_t)cnt[1];
    st->columns += (int64_t)cnt[2];
  }
  return 0;
}

static int reset_stats(xtg_ctx *c) {
  CK(cudaMemsetAsync(c->d_absx, 0, NSLOT * 8, c->st));
  CK(cudaMemsetAsync(c->d_cnt, 0, 3 * 8, c->st));
  return 0;
}

// Reference-order random lists (randomly_select_x_y, XT_ICD_update.c:599-631)
// drawn with the reference generator, for the sequential parity mode.
static void host_random_lists(xtg_ctx *c, std::vector<int> &usn, std::vector<int> &xs, std::vector<int> &ys) {
  const xt_geom &g = c->g;
  const int nxy = (int)c->nxy;
  usn.assign((size_t)g.N_time * g.nzb, 0);
  xs.assign((size_t)g.N_time * g.nzb * nxy, 0);
  ys.assign((size_t)g.N_time * g.nzb * nxy, 0);
  std::vector<int> counter(nxy);
  for (int i = 0; i < g.N_time; i++)
    for (int b = 0; b < g.nzb; b++) {
      int size = nxy;
      int &u = usn[(size_t)i * g.nzb + b];
      for (int q = 0; q < nxy; q++) counter[q] = q;
      for (int jj = 0; jj < nxy; jj++) {
        int index = (int)floor(rng_next(c) * size);
        index = (index == size) ? size - 1 : index;
        const int col = counter[index] % g.N_x, row = counter[index] / g.N_x;
        if (c->col_rank[(size_t)row * g.N_x + col] >= 0) {
          xs[((size_t)i * g.nzb + b) * nxy + u] = col;
          ys[((size_t)i * g.nzb + b) * nxy + u] = row;
          u++;
        }
        counter[index] = counter[size - 1];
        size--;
      }
    }
}

// RandomizedSelect with the reference generator (XT_NHICD.c:63-126), used in
// the sequential mode so later iterations draw the reference's numbers.
static float host_randomized_select(xtg_ctx *c, float *A, unsigned p, unsigned r, unsigned i) {
  for (;;) {
    if (p == r) return A[p];
    unsigned rnum = (unsigned)floor(rng_next(c) * (r - p + 1));
    rnum = (rnum == r - p + 1) ? r - p : rnum;
    const unsigned j = p + rnum;
    std::swap(A[r], A[j]);
    const float x = A[r];
    unsigned ii = p - 1;
    for (unsigned jj = p; jj < r; jj++)
      if (A[jj] <= x) {
        ii++;
        std::swap(A[ii], A[jj]);
      }
    std::swap(A[ii + 1], A[r]);
    const unsigned q = ii + 1, k = q - p + 1;
    if (i == k) return A[q];
    if (i < k)
      r = q - 1;
    else {
      p = q + 1;
      i -= k;
    }
  }
}

// Halo exchange of a z slab (the reference's MPI_Send_Recv_Z_Slices /
// MPI_Wait_Z_Slices after every half-pass, XT_MPI.c:47-122): this slab's
// boundary slices go into the send planes, the stream is drained, and the
// caller's hook moves them to the neighbours and fills the halo planes
// before the next launch reads them.
static int slab_exchange(xtg_ctx *c) {
  if (!c->xfn) return 0;
  if (c->send_lo || c->send_hi) {
    const size_t n = (size_t)c->g.N_time * c->g.N_y * c->g.N_x;
    k_slab_pack<<<std::min<unsigned>(blocks_for(n, 256), (unsigned)c->sm_count * 4), 256, 0, c->st>>>(
        c->G, c->d_x, c->send_lo, c->send_hi);
    c->launches++;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->st));
  const int rc = c->xfn(c->xuser, c->xphase++);
  if (rc) {
    set_err("slab halo exchange hook failed (%d)", rc);
    return XTG_E_STATE;
  }
  return 0;
}

static int icd_iteration_parallel(xtg_ctx *c, int iter, xtg_stats *st) {
  const long long icd0 = c->icd_launches;
  const xt_geom &g = c->g;
  const int n = g.N_time * c->n_masked;
  const unsigned long long key = c->seed * 0x9E3779B97F4A7C15ULL + (unsigned long long)iter * 0xD1B54A32D192ED03ULL;
  k_build_items<<<blocks_for(n, 256), 256, 0, c->st>>>(n, c->n_masked, g.N_x, c->d_mcols, key, c->d_items);
  c->launches++;
  CK(cudaGetLastError());
  const int K = XT_NHICD_CHUNKS, chunk = n / K;
  const int cap0 = (int)(c->nh_cap / 2);
  float kms_total = 0.f;
  long long items_total = 0;
  double vox_mag = 0;
  // ICD launches are timed with event pairs read once at the end of the
  // iteration, so the host never waits between launches
  const size_t npair = (size_t)3 * K;
  while (c->tev.size() < 2 * npair) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    c->tev.push_back(e);
  }
  size_t ntimed = 0;
  for (int j = 0; j < K; j++) {
    const int lo = j * chunk, hi = (j == K - 1) ? n : (j + 1) * chunk;
    if (j == K - 1) {  // the reference's vox_mag covers the last chunk only (XT_ICD_update.c:798)
      double tmp;
      int rc = read_stats(c, st, &tmp);
      if (rc) return rc;
      rc = reset_stats(c);
      if (rc) return rc;
    }
    CK(cudaEventRecord(c->tev[2 * ntimed], c->st));
    int rc = run_columns(c, iter, c->d_items, lo, hi - lo, nullptr, 0, 0, 1, 0, -1);
    if (rc) return rc;
    CK(cudaEventRecord(c->tev[2 * ntimed + 1], c->st));
    ntimed++;
    if ((rc = slab_exchange(c))) return rc;
    if (j == K - 1) {
      rc = read_stats(c, st, &vox_mag);
      if (rc) return rc;
      rc = reset_stats(c);
      if (rc) return rc;
    }
    items_total += hi - lo;
    if (c->prm.updateProjOffset > 1) {
      rc = xtg_update_offset(c);
      if (rc) return rc;
    }
    rc = nhicd_select_device(c);
    if (rc) return rc;
    if (iter > 1 && !c->prm.no_NHICD) {
      for (int h = 0; h < 2; h++) {
        CK(cudaEventRecord(c->tev[2 * ntimed], c->st));
        rc = run_columns(c, iter, c->d_nh, h ? cap0 : 0, 0, c->d_nhcnt + h, 1, key + 17 * (j * 2 + h + 1), 0, 1, -1);
        if (rc) return rc;
        CK(cudaEventRecord(c->tev[2 * ntimed + 1], c->st));
        ntimed++;
        if ((rc = slab_exchange(c))) return rc;
        if (c->prm.updateProjOffset > 1) {
          rc = xtg_update_offset(c);
          if (rc) return rc;
        }
      }
    }
  }
  if (ntimed) CK(cudaEventSynchronize(c->tev[2 * ntimed - 1]));
  for (size_t i = 0; i < ntimed; i++) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
    kms_total += ms;
  }
  double tmp;
  int rc = read_stats(c, st, &tmp);
  if (rc) return rc;
  c->last_kms = kms_total;
  c->last_items = items_total;
  c->last_icd = c->icd_launches - icd0;
  st->vox_mag = vox_mag;
  return 0;
}

static int icd_iteration_sequential(xtg_ctx *c, int iter, xtg_stats *st) {
  const long long icd0 = c->icd_launches;
  const xt_geom &g = c->g;
  const int nxy = (int)c->nxy, K = XT_NHICD_CHUNKS;
  std::vector<int> usn, xs, ys;
  host_random_lists(c, usn, xs, ys);
  std::vector<int4> items;
  double vox_mag = 0;
  float kms_total = 0;
  long long items_total = 0;
  auto run_list = [&](std::vector<int4> &L) -> int {
    if (L.empty()) return 0;
    if (L.size() > c->items_cap) {
      set_err("work list too long");
      return XTG_E_ARG;
    }
    CK(cudaMemcpyAsync(c->d_items, L.data(), L.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    CK(cudaEventRecord(c->ek0, c->st));
    int rc = run_columns(c, iter, c->d_items, 0, (int)L.size(), nullptr, 0, 0, 0, 1, 1);
    if (rc) return rc;
    CK(cudaEventRecord(c->ek1, c->st));
    CK(cudaEventSynchronize(c->ek1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ek0, c->ek1));
    kms_total += ms;
    items_total += (long long)L.size();
    return 0;
  };
  std::vector<float> filt((size_t)nxy), filtc((size_t)nxy);
  std::vector<int> nsn((size_t)g.N_time * g.nzb);
  std::vector<int> xn((size_t)g.N_time * g.nzb * nxy), yn((size_t)g.N_time * g.nzb * nxy);
  for (int j = 0; j < K; j++) {
    if (j == K - 1) {
      double tmp;
      int rc = read_stats(c, st, &tmp);
      if (rc) return rc;
      rc = reset_stats(c);
      if (rc) return rc;
    }
    for (int half = 0; half < 2; half++) {
      items.clear();
      for (int i = 0; i < g.N_time; i++)
        for (int b = 0; b < g.nzb; b += 2) {
          const int idx = (((i % 2) == 0) ^ half) ? b : b + 1;
          const int u = usn[(size_t)i * g.nzb + idx];
          const int xb = j * (int)floor(u / K);
          const int xe = (j == K - 1) ? u - 1 : (j + 1) * (int)floor(u / K) - 1;
          for (int q = xb; q <= xe; q++)
            items.push_back(make_int4(i, ys[((size_t)i * g.nzb + idx) * nxy + q], xs[((size_t)i * g.nzb + idx) * nxy + q], idx));
        }
      int rc = run_list(items);
      if (rc) return rc;
      if (c->prm.updateProjOffset > 1) {
        rc = xtg_update_offset(c);
        if (rc) return rc;
      }
    }
    if (j == K - 1) {
      int rc = read_stats(c, st, &vox_mag);
      if (rc) return rc;
      rc = reset_stats(c);
      if (rc) return rc;
    }
    // NHICD selection with the reference's RandomizedSelect on the device-filtered map
    const int nseg = g.N_time * g.nzb;
    const unsigned grid = std::min<unsigned>(blocks_for(c->nmag, 256), (unsigned)c->sm_count * 8);
    k_vsc_filter<<<grid, 256, 0, c->st>>>(nseg, g.N_y, g.N_x, c->d_mag, c->d_filt);
    c->launches++;
    std::vector<float> allf(c->nmag);
    CK(cudaMemcpyAsync(allf.data(), c->d_filt, c->nmag * 4, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int s = 0; s < nseg; s++) {
      const int n = (int)floor(usn[s] / XT_NHICD_CHUNKS);
      memcpy(filt.data(), &allf[(size_t)s * nxy], (size_t)nxy * 4);
      memcpy(filtc.data(), filt.data(), (size_t)nxy * 4);
      const float th = host_randomized_select(c, filt.data(), 0, (unsigned)(nxy - 1), (unsigned)(nxy - n));
      int idx = 0;
      for (int r = 0; r < g.N_y; r++)
        for (int k = 0; k < g.N_x; k++)
          if (filtc[(size_t)r * g.N_x + k] > th) {
            xn[(size_t)s * nxy + idx] = k;
            yn[(size_t)s * nxy + idx] = r;
            idx++;
          }
      nsn[s] = idx;
    }
    if (iter > 1 && !c->prm.no_NHICD) {
      for (int half = 0; half < 2; half++) {
        items.clear();
        for (int i = 0; i < g.N_time; i++)
          for (int b = 0; b < g.nzb; b += 2) {
            const int idx = (((i % 2) == 0) ^ half) ? b : b + 1;
            const int s = i * g.nzb + idx;
            for (int q = 0; q < nsn[s]; q++) {
              const int yy = yn[(size_t)s * nxy + q], xx = xn[(size_t)s * nxy + q];
              // a selected column outside the support disk has no voxel to update
              if (c->col_rank[(size_t)yy * g.N_x + xx] >= 0) items.push_back(make_int4(i, yy, xx, idx));
            }
          }
        int rc = run_list(items);
        if (rc) return rc;
        if (c->prm.updateProjOffset > 1) {
          rc = xtg_update_offset(c);
          if (rc) return rc;
        }
      }
    }
  }
  double tmp;
  int rc = read_stats(c, st, &tmp);
  if (rc) return rc;
  c->last_kms = kms_total;
  c->last_items = items_total;
  c->last_icd = c->icd_launches - icd0;
  st->vox_mag = vox_mag;
  return 0;
}

int xtg_icd_iteration(xtg_ctx *c, int32_t iter, xtg_stats *st_out) {
  if (!c) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_icd_iteration: no sinogram uploaded");
    return XTG_E_STATE;
  }
  xtg_stats st;
  memset(&st, 0, sizeof(st));
  int rc = reset_stats(c);
  if (rc) return rc;
  // a slab starts every iteration from its neighbours' current boundary slices
  c->xphase = 0;
  if ((rc = slab_exchange(c))) return rc;
  CK(cudaEventRecord(c->ev0, c->st));
  rc = (c->order == XTG_ORDER_SEQUENTIAL) ? icd_iteration_sequential(c, iter, &st) : icd_iteration_parallel(c, iter, &st);
  if (rc) return rc;
  if (c->prm.do_VarEst) {
    rc = xtg_update_variance(c);
    if (rc) return rc;
  }
  // stop statistic (XT_ICD_update.c:884-925)
  CK(cudaMemsetAsync(c->d_red + 4 * NSLOT, 0, NSLOT * 8, c->st));
  magsum_launch(c);
  CK(cudaGetLastError());
  double h[NSLOT];
  CK(cudaMemcpyAsync(h, c->d_red + 4 * NSLOT, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaEventRecord(c->ev1, c->st));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(&st.ms, c->ev0, c->ev1));
  double ms = 0;
  for (int i = 0; i < NSLOT; i++) ms += h[i];
  st.mag_sum = ms;
  st.total_pix = (double)c->n_masked * c->g.N_time * c->g.nzb * (double)(c->g.N_z / c->g.nzb);
  st.avg_update_pct = (st.vox_mag > 0) ? 100.0 * ms / st.vox_mag : INFINITY;
  st.converged = st.avg_update_pct < (double)c->g.StopThreshold;
  rc = check_err_flag(c);
  if (rc) return rc;
  if (st_out) *st_out = st;
  return 0;
}

int xtg_update_columns(xtg_ctx *c, int32_t iter, int32_t n, const int32_t *items, xtg_stats *st_out) {
  if (!c) return XTG_E_ARG;
  const long long icd0 = c->icd_launches;
  if (!c || n < 0 || (n && !items)) return XTG_E_ARG;
  if (!c->have_sino) {
    set_err("xtg_update_columns: no sinogram uploaded");
    return XTG_E_STATE;
  }
  if ((size_t)n > c->items_cap) {
    set_err("xtg_update_columns: %d items exceed the list capacity %zu", n, c->items_cap);
    return XTG_E_ARG;
  }
  const xt_geom &g = c->g;
  int any_whole = 0, any_block = 0;
  for (int q = 0; q < n; q++) {
    const int f = items[4 * q], r = items[4 * q + 1], k = items[4 * q + 2], b = items[4 * q + 3];
    if (f < 0 || f >= g.N_time || r < 0 || r >= g.N_y || k < 0 || k >= g.N_x || b < -1 || b >= g.nzb) {
      set_err("xtg_update_columns: item %d out of range", q);
      return XTG_E_ARG;
    }
    if (c->a_mode != XTG_A_FP32 && c->col_rank[(size_t)r * g.N_x + k] < 0) {
      set_err("xtg_update_columns: the A table covers masked columns only (item %d)", q);
      return XTG_E_ARG;
    }
    if (b >= 0) any_block = 1; else any_whole = 1;
  }
  xtg_stats st;
  memset(&st, 0, sizeof(st));
  int rc = reset_stats(c);
  if (rc) return rc;
  if (n) CK(cudaMemcpyAsync(c->d_items, items, (size_t)n * sizeof(int4), cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->ek0, c->st));
  rc = run_columns(c, iter, c->d_items, 0, n, nullptr, 0, 0, any_whole, any_block, -1);
  if (rc) return rc;
  CK(cudaEventRecord(c->ek1, c->st));
  double ab = 0;
  rc = read_stats(c, &st, &ab);
  if (rc) return rc;
  CK(cudaEventElapsedTime(&st.ms, c->ek0, c->ek1));
  st.vox_mag = ab;
  c->last_kms = st.ms;
  c->last_items = n;
  c->last_icd = c->icd_launches - icd0;
  rc = check_err_flag(c);
  if (rc) return rc;
  if (st_out) *st_out = st;
  return 0;
}

int xtg_nhicd_select(xtg_ctx *c, const int32_t *usn, int32_t *nnum, int32_t *xsel, int32_t *ysel, float *thr) {
  if (!c || !usn || !nnum) return XTG_E_ARG;
  const xt_geom &g = c->g;
  const int nseg = g.N_time * g.nzb;
  std::vector<int> kth(nseg);
  for (int s = 0; s < nseg; s++) kth[s] = (int)c->nxy - (int)floor(usn[s] / XT_NHICD_CHUNKS);
  for (int s = 0; s < nseg; s++)
    if (kth[s] < 1 || kth[s] > (int)c->nxy) {
      set_err("xtg_nhicd_select: update_select_num out of range");
      return XTG_E_ARG;
    }
  CK(cudaMemcpyAsync(c->d_kth, kth.data(), nseg * 4, cudaMemcpyHostToDevice, c->st));
  const unsigned grid = std::min<unsigned>(blocks_for(c->nmag, 256), (unsigned)c->sm_count * 8);
  k_vsc_filter<<<grid, 256, 0, c->st>>>(nseg, g.N_y, g.N_x, c->d_mag, c->d_filt);
  radix_select_multi(c, nseg);
  c->launches += 1;
  CK(cudaGetLastError());
  std::vector<float> th(nseg), f(c->nmag);
  CK(cudaMemcpyAsync(th.data(), c->d_thr, nseg * 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(f.data(), c->d_filt, c->nmag * 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  // lists in the reference's raster order
  for (int s = 0; s < nseg; s++) {
    int idx = 0;
    for (int r = 0; r < g.N_y; r++)
      for (int k = 0; k < g.N_x; k++)
        if (f[(size_t)s * c->nxy + (size_t)r * g.N_x + k] > th[s]) {
          if (xsel) xsel[(size_t)s * c->nxy + idx] = k;
          if (ysel) ysel[(size_t)s * c->nxy + idx] = r;
          idx++;
        }
    nnum[s] = idx;
    if (thr) thr[s] = th[s];
  }
  return 0;
}

int64_t xtg_device_bytes(const xtg_ctx *c) { return c ? (int64_t)c->dev_bytes : 0; }
int64_t xtg_launch_count(const xtg_ctx *c) { return c ? (int64_t)c->launches : 0; }

int xtg_last_kernel_time(const xtg_ctx *c, float *ms, int64_t *items, int64_t *launches) {
  if (!c) return XTG_E_ARG;
  if (ms) *ms = c->last_kms;
  if (items) *items = c->last_items;
  if (launches) *launches = c->last_icd;
  return 0;
}

}  // extern "C"

// ------------------------------------------- allocation-free NHICD threshold --
// Scratch of xtg_nhicd_threshold_noalloc: the filtered maps, then the per-map
// ranks.  It lives for the life of the library on every device that loads it.
// Host code must not use the symbol itself as a device address (it is a host
// stand-in); the device address comes from cudaGetSymbolAddress, once per
// device.
static __device__ __align__(256) float g_noalloc_scratch[XTG_NOALLOC_MAX_ELEMS + XTG_NOALLOC_MAX_MAPS];

struct NoallocRanks {
  int k[XTG_NOALLOC_MAX_MAPS];
};

// the ranks travel by value in the launch, so no host-to-device copy (and no
// staging allocation) is needed
__global__ void k_noalloc_put_ranks(NoallocRanks r, int n, int *dst) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = r.k[i];
}

__global__ void k_noalloc_select(size_t n, int plane, const float *filt, const float *thr, unsigned char *sel) {
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    sel[q] = filt[q] > thr[q / plane] ? 1 : 0;
}

static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[256];

extern "C" int xtg_nhicd_threshold_noalloc(const float *magmap, int32_t nmaps, int32_t ny, int32_t nx,
                                           const int32_t *kth, float *thresholds, uint8_t *select, void *stream) {
  if (!magmap || !kth || !thresholds || nmaps < 1 || ny < 1 || nx < 1) {
    set_err("xtg_nhicd_threshold_noalloc: null pointer or empty map");
    return XTG_E_ARG;
  }
  const size_t plane = (size_t)ny * nx, n = (size_t)nmaps * plane;
  if (n > (size_t)XTG_NOALLOC_MAX_ELEMS || nmaps > XTG_NOALLOC_MAX_MAPS) {
    set_err("xtg_nhicd_threshold_noalloc: %d maps of %d x %d (%zu values) exceed the fixed scratch of %d values "
            "in at most %d maps; use xtg_nhicd_select instead",
            nmaps, ny, nx, n, XTG_NOALLOC_MAX_ELEMS, XTG_NOALLOC_MAX_MAPS);
    return XTG_E_ARG;
  }
  NoallocRanks r;
  for (int s = 0; s < nmaps; s++) {
    if (kth[s] < 1 || (size_t)kth[s] > plane) {
      set_err("xtg_nhicd_threshold_noalloc: rank %d of map %d outside 1..%zu", kth[s], s, plane);
      return XTG_E_ARG;
    }
    r.k[s] = kth[s];
  }
  // an error left by the caller's own earlier work is reported as such and
  // left pending for the caller, not taken for one of the launches below
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    set_err("xtg_nhicd_threshold_noalloc: a CUDA error from earlier work is pending: %s",
            cudaGetErrorString(pending));
    return XTG_E_CUDA;
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) {
    set_err("xtg_nhicd_threshold_noalloc: device ordinal %d out of range", dev);
    return XTG_E_ARG;
  }
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {  // first call on this device: resolve the array's device address
      CK(cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch));
    }
    base = g_noalloc_addr[dev];
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  float *filt = reinterpret_cast<float *>(base);
  int *ranks = reinterpret_cast<int *>(filt + XTG_NOALLOC_MAX_ELEMS);
  // every value read below is written first in this call: no clearing needed
  k_noalloc_put_ranks<<<1, 256, 0, st>>>(r, nmaps, ranks);
  CK(cudaGetLastError());
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 4096);
  k_vsc_filter<<<grid, 256, 0, st>>>(nmaps, ny, nx, magmap, filt);
  CK(cudaGetLastError());
  k_radix_select<<<nmaps, 1024, 0, st>>>(filt, (int)plane, ranks, thresholds);
  CK(cudaGetLastError());
  if (select) {
    k_noalloc_select<<<grid, 256, 0, st>>>(n, (int)plane, filt, thresholds, select);
    CK(cudaGetLastError());
  }
  return 0;
}
