// xtg_icd.cu -- the ICD column kernel: one CTA updates one x-y column's
// z-line (or one z-block of it) of one time frame.
//
// Parallel-beam A is z-invariant: every slice of a column sees the same
// (view, bin) entries, and the rows of slice z are t = z*zovl .. z*zovl+zovl-1.
// So the CTA puts the column's A into shared memory once (computed in
// registers, or read from the FP16 table), then streams the column's
// footprint e[p][bin][t0..t0+T) and w[...] (contiguous in t) with 16-byte
// loads, thread (view group, t lane) accumulating theta1/theta2 for its rows;
// shuffles and one shared-memory pass reduce them over view groups.  The
// slices' qGGMRF surrogate steps run in red/black z order with 8 lanes per
// voxel (or strictly in increasing z on one thread, the reference's order, in
// sequential mode), and the e update goes back with vector red.global.add,
// so columns in flight that share sinogram entries never lose an update.
//
// Reference: updateVoxels_Aditya + compute_voxel_update_Aditya
// (Source_Code_4D_Fast/XT_VoxUpdate.c:11-254), CE_FunctionalSubstitution
// (XT_ICD_update.c:130-179); the z-line batching follows updateVoxels_AttTomo
// (XT_VoxUpdate.c:266-586).
#include "xtg_internal.h"

namespace xtg {

// Work items of at most XTG_SMALL_ROWS detector rows run in CTAs of
// XTG_SMALL_NT threads (table modes, parallel schedule).
#ifndef XTG_SMALL_ROWS
#define XTG_SMALL_ROWS 16
#endif
#ifndef XTG_SMALL_NT
#define XTG_SMALL_NT 64
#endif
// Longer items whose column runs hold at most XTG_MEDIUM_ENTRIES A entries
// run in CTAs of XTG_MEDIUM_NT threads (table modes, parallel schedule): the
// per-item fixed work weighs more when the footprint is short, and twice as
// many CTAs per SM overlap it better.  The largest 4D volume (352 entries
// per column and frame): 745 -> 888 M voxel updates/s; 64 threads: equal;
// plain 3D (2195 entries) in 128-thread CTAs: 221 against 241 M.
#ifndef XTG_MEDIUM_ENTRIES
#define XTG_MEDIUM_ENTRIES 1024
#endif
#ifndef XTG_MEDIUM_NT
#define XTG_MEDIUM_NT 128
#endif

// Footprint loads with L2 cache hints: e (re-read and updated through L2 by
// other columns' reductions) is kept (evict_last), w (read once per visit) is
// evicted first; neither is allocated in L1.
__device__ __forceinline__ float4 ld_e(const float *p) {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  float4 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_w(const float *p, bool keep) {
  uint64_t pol;
  if (keep)  // e and w fit in L2 together: keep w as well
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  else
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  float4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p), "l"(pol));
  return v;
}

// Asynchronous global -> shared copies (no registers held while in flight);
// cp_wait_all completes the calling thread's copies and makes them visible to it.
__device__ __forceinline__ uint32_t icd_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void *s, const void *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(icd_smem(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(void *s, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(icd_smem(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(void *s, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(icd_smem(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Where a work item's column run lies in the A column table, fetched for the
// next item while the current one is processed (small CTAs).
struct ItemMeta {
  int4 item;           // frame, row, column, z-block
  long long s0, s1;    // tstart[ti], tstart[ti + 1]
  float sc;            // tscale[ti] (FP16 table)
  int rank;            // col_rank[row][column]
  int it;              // launch-wide item index (>= the launch's total: none)
  int pad;
};

// Packed FP32 (two lanes per instruction, sm_100) for the footprint
// arithmetic of 16-byte rows
#ifndef XTG_F32X2
#define XTG_F32X2 1
#endif

// Footprint entries a thread loads before it uses any of them (table modes,
// 16-byte rows): more loads in flight per warp to cover L2/HBM latency.
// Three measured equal in the 256-thread CTAs (a few bytes spilled) and 1 %
// slower in the 64-thread ones, which keep two whatever this is set to.
#ifndef XTG_UNROLL
#define XTG_UNROLL 2
#endif

// surrogate coefficient with fast intrinsics: the step size only needs a few
// digits, the fixed point of the iteration is unchanged
__device__ __forceinline__ float qcoef_fast(float d, float sq, float sqp, float c, float p) {
  if (d == 0.f) return __fdividef(2.0f, sq * c);
  const float t1 = __fdividef(__powf(fabsf(d), 2.0f - p), sqp);
  const float t3 = c + t1;
  return __fdividef(2.0f - __fdividef((2.0f - p) * t1, t3), t3 * sq);
}

// the 29 neighbour slots of a voxel: 0..26 the 3x3x3 block in [dz][dy][dx]
// order (13 = the voxel itself, skipped), 27 = frame - 1, 28 = frame + 1
struct Nbr {
  float v;
  float b;  // filter weight * surrogate coefficient, 0 when the slot is absent
};

// hlo / hhi: the slices below slice 0 and above slice N_z - 1 belong to a
// neighbouring slab (their values are staged in sNb like any other)
__device__ __forceinline__ Nbr nbr_term(const DevGeo &G, const float *sNb, const float *sTn, int zmax, int z, int zb,
                                        int fr, int row, int col, float Vv, int n, bool hlo, bool hhi) {
  Nbr o{0.f, 0.f};
  if (n < 27) {
    if (n == 13) return o;
    const int dz = n / 9, c = n % 9;
    const int za = zb + z + dz - 1;
    if ((za < 0 && !hlo) || (za >= G.N_z && !hhi)) return o;
    const int jj = row + c / 3 - 1, kk = col + c % 3 - 1;
    if (jj < 0 || jj >= G.N_y || kk < 0 || kk >= G.N_x) return o;
    o.v = sNb[c * (zmax + 2) + z + dz];
    o.b = G.SF[n] * qcoef_fast(Vv - o.v, G.Sigma_S_Q, G.Sigma_S_Q_P, G.C_S, G.MRF_P);
  } else {
    const int f2 = fr + (n == 27 ? -1 : 1);
    if (f2 < 0 || f2 >= G.N_time) return o;
    o.v = sTn[(n - 27) * zmax + z];
    o.b = G.TF * qcoef_fast(Vv - o.v, G.Sigma_T_Q, G.Sigma_T_Q_P, G.C_T, G.MRF_P);
  }
  return o;
}

// Next-item prefetch in the 256-thread CTAs too (the small ones always):
// measured equal on plain 3D (237.6-238.5 against 236.5-237.1 M voxel
// updates/s), so off
#ifndef XTG_PF_ALL
#define XTG_PF_ALL 0
#endif

// resident 256-thread CTAs per SM the register budget is cut for (5: 48
// registers with spills, 8 % slower on plain 3D)
#ifndef XTG_CTAS_256
#define XTG_CTAS_256 4
#endif

// NT threads per CTA: 256 for long z-lines; 64 where a work item is short
// (few detector rows), so the per-item fixed work (neighbourhood, A staging,
// barriers, the surrogate step) runs in four times as many CTAs at once.
template <int VEC, int AMODE, int SEQ, int AS, int NT = XTG_THREADS>
__global__ void __launch_bounds__(NT, NT == XTG_THREADS ? XTG_CTAS_256 : 1024 / NT) k_icd_columns(DevGeo G, IcdArgs A, int vmax,
                                                                                 int zmax) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NW = NT / 32;
  unsigned char *smem = smem_raw;
  // AMODE 0 (A computed here): per view {first | n << 24, view index, AS values}
  int *sPack = reinterpret_cast<int *>(smem);            // [vmax]
  int *sView = sPack + vmax;                              // [vmax]
  float *sVal = reinterpret_cast<float *>(sView + vmax);  // [AS][vmax] A * delta_t
  // AMODE 1/2 (column table): the column's entry run, vmax = longest run,
  // {(p*N_r + bin)*N_t, bits of A * delta_t} per entry (one 8-byte load)
  int2 *sEnt = reinterpret_cast<int2 *>(smem);           // [vmax]
  float *sRed = (AMODE == 0) ? sVal + (size_t)vmax * AS : reinterpret_cast<float *>(sEnt + vmax);  // [2][NW][128]
  float *sTh = sRed + 2 * NW * 128;                       // [2][zmax*zovl]
  const int rowsmax = zmax * G.zovl;
  float *sNb = sTh + 2 * rowsmax;                         // [9][zmax+2]
  float *sTn = sNb + 9 * (zmax + 2);                      // [2][zmax]
  float *sDelta = sTn + 2 * zmax;                         // [zmax]

  __shared__ int sItem;
  __shared__ double sAbs[NT / 32];
  __shared__ unsigned sUpd, sZero;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nitems = A.n_items_dev ? *A.n_items_dev : A.n_items;
  const bool hlo = A.halo_lo != nullptr, hhi = A.halo_hi != nullptr;
  // Short items (small CTAs) are taken GRAB at a time and the CTA's
  // statistics are added up in thread 0 and flushed once at the end: with
  // tens of thousands of items per launch, per-item atomics on the same few
  // addresses would queue at L2.
  // (kept in shared memory: registers are the kernel's occupancy limit)
  constexpr int GRAB = NT < XTG_THREADS ? 8 : 1;
  __shared__ int sGrab[2];                 // base, next of the batch
  __shared__ double sCtaAbs;
  __shared__ unsigned long long sCta[3];   // voxel updates, zero skipped, items
  // Small CTAs fetch the next item's record and table run asynchronously in
  // three dependent steps (record; column rank; run bounds), one per phase of
  // the current item, so that the chain's round trips overlap its work.
  constexpr bool PF = (NT < XTG_THREADS || XTG_PF_ALL) && AMODE != 0 && !SEQ;
  __shared__ __align__(16) ItemMeta sMeta[2];
  int mb = 0;  // sMeta[mb]: the current item; sMeta[mb ^ 1]: the next
  const int total = nitems * A.nsub;
  auto grab = [&]() -> int {  // thread 0 only
    if (sGrab[1] == GRAB) {
      sGrab[0] = atomicAdd(A.counter, GRAB);
      sGrab[1] = 0;
    }
    return sGrab[0] + sGrab[1]++;
  };
  auto item_index = [&](int i) -> int {
    const int ii = A.nsub == 1 ? i : i % nitems;
    return A.item_lo + (A.use_perm ? (int)xt_perm((uint32_t)ii, (uint32_t)nitems, A.perm_key) : ii);
  };
  auto fetch_rank = [&]() {  // thread 0, the next item's record in place
    ItemMeta &N = sMeta[mb ^ 1];
    if (N.it < total) cp_async4(&N.rank, A.col_rank + N.item.y * G.N_x + N.item.z);
  };
  auto fetch_bounds = [&]() {  // thread 0, the next item's rank in place
    ItemMeta &N = sMeta[mb ^ 1];
    if (N.it < total) {
      const long long ti = (long long)N.item.x * A.n_masked + N.rank;
      cp_async8(&N.s0, A.tstart + ti);
      cp_async8(&N.s1, A.tstart + ti + 1);
      if (AMODE == 1) cp_async4(&N.sc, A.tscale + ti);
    }
  };
  // the rank and run-bound steps with plain loads (prologue, skipped pieces)
  auto meta_finish = [&](ItemMeta &N) {
    if (N.it >= total) return;
    N.rank = A.col_rank[N.item.y * G.N_x + N.item.z];
    const long long ti = (long long)N.item.x * A.n_masked + N.rank;
    N.s0 = A.tstart[ti];
    N.s1 = A.tstart[ti + 1];
    N.sc = (AMODE == 1) ? A.tscale[ti] : 1.f;
  };
  if (tid == 0) {
    sGrab[0] = 0;
    sGrab[1] = GRAB;
    sCtaAbs = 0.0;
    sCta[0] = sCta[1] = sCta[2] = 0;
    if (PF) {
      sMeta[0].it = grab();
      if (sMeta[0].it < total) {
        sMeta[0].item = A.items[item_index(sMeta[0].it)];
        meta_finish(sMeta[0]);
      }
    }
  }

  for (;;) {
    if (tid == 0) {
      if (PF) {
        ItemMeta &N = sMeta[mb ^ 1];
        N.it = grab();
        if (N.it < total) cp_async16(&N.item, A.items + item_index(N.it));
      } else {
        sItem = grab();
      }
      sUpd = 0;
      sZero = 0;
    }
    __syncthreads();
    const int it = PF ? sMeta[mb].it : sItem;
    if (it >= total) break;
    const int piece = A.nsub == 1 ? 0 : it / nitems;
    const int4 item = PF ? sMeta[mb].item : A.items[item_index(it)];
    const int fr = item.x, row = item.y, col = item.z, blk = item.w;
    int zb = 0, ze = G.N_z - 1;
    if (blk >= 0) {
      zb = blk * G.zstep;
      ze = (blk >= G.nzb - 1) ? G.N_z - 1 : (blk + 1) * G.zstep - 1;
    }
    zb += piece * A.zslab;
    if (zb > ze) {  // this item has fewer pieces (uniform over the CTA)
      if (PF && tid == 0) {
        cp_wait_all();
        meta_finish(sMeta[mb ^ 1]);
      }
      __syncthreads();
      mb ^= 1;
      continue;
    }
    ze = min(ze, zb + A.zslab - 1);
    const int Z = ze - zb + 1, T = Z * G.zovl, t0 = zb * G.zovl;
    const int V = A.view_num[fr], vs = A.view_start[fr];

    // 1. neighbourhood: the 3x3 columns' z-lines over [zb-1, ze+1], and the
    //    same column in frames fr-1 and fr+1 (0 outside the volume; slices
    //    -1 and N_z from the neighbouring slabs' halo planes when present,
    //    as the reference's ranks read Object[i][0] / [N_z+1],
    //    XT_VoxUpdate.c:94-99)
    const size_t plane = (size_t)G.N_y * G.N_x;
    // (small CTAs, FP32 table) the column's table run goes to shared memory
    // asynchronously first, so that its round trip overlaps the
    // neighbourhood's; a quiet line (below) has fetched it for nothing
    constexpr bool PFE = PF && AMODE == 2;
    if (PFE) {
      const long long s0 = sMeta[mb].s0;
      const int n = (int)(sMeta[mb].s1 - s0);
      for (int e = tid; e < n; e += NT) {
        cp_async4(&sEnt[e].x, A.toff + s0 + e);
        cp_async4(&sEnt[e].y, A.tval32 + s0 + e);
      }
    }
    // Zero skipping (XT_VoxUpdate.c:208-232) decided for the whole z-line
    // before any footprint work: from the second iteration a voxel equal to 0
    // with no positive spatial or temporal neighbour is not updated.  When
    // that holds for every voxel of the item, theta is never used, so neither
    // A nor the footprint is read (the update step below skips each voxel by
    // the same test and the e update has nothing to add).  Each thread tests
    // the values it stages.
    bool quiet = A.iter > 1;
    // k / (Z + 2) as (k * mz2) >> 20: exact while k (Z + 2) < 2^20, and here
    // k < 9 (Z + 2) with Z + 2 <= 130
    const uint32_t z2 = (uint32_t)Z + 2u, mz2 = ((1u << 20) + z2 - 1u) / z2;
    for (int k = tid; k < 9 * (Z + 2); k += NT) {
      const int c = (int)(((uint32_t)k * mz2) >> 20), zz = k - c * (Z + 2);
      const int jj = row + c / 3 - 1, kk = col + c % 3 - 1, za = zb - 1 + zz;
      float v = 0.f;
      if (jj >= 0 && jj < G.N_y && kk >= 0 && kk < G.N_x) {
        const size_t q = (size_t)fr * plane + (size_t)jj * G.N_x + kk;
        if (za >= 0 && za < G.N_z)
          v = A.x[q * G.N_z + za];
        else if (za < 0 && hlo)
          v = A.halo_lo[q];
        else if (za >= G.N_z && hhi)
          v = A.halo_hi[q];
      }
      sNb[c * (zmax + 2) + zz] = v;
      const bool self = (c == 4) && zz >= 1 && zz <= Z;
      if (self ? (v != 0.f) : (v > 0.f)) quiet = false;
    }
    for (int k = tid; k < 2 * Z; k += NT) {
      const int s = k >= Z ? 1 : 0, z = k - s * Z, f2 = fr + (s ? 1 : -1);
      float v = 0.f;
      if (f2 >= 0 && f2 < G.N_time) v = A.x[(((size_t)f2 * plane) + (size_t)row * G.N_x + col) * G.N_z + zb + z];
      sTn[s * zmax + z] = v;
      if (v > 0.f) quiet = false;
    }
    const bool skip_all = __syncthreads_and(quiet) != 0;
    // 2. the column's A entries (times delta_t, XT_VoxUpdate.c:27) -> smem
    if (AMODE == 0 && !skip_all) {
      for (int v = tid; v < V; v += NT) {
        const int p = A.view_idx[vs + v];
        float vals[AS];
        int first;
        const int n = xt_amatrix_regs<AS>(G, A.hr + (size_t)p * XT_HR_STRIDE, A.cosv[p], A.sinv[p], row, col, vals,
                                          &first);
        sPack[v] = first | (n << 24);
        sView[v] = p;
#pragma unroll
        for (int s = 0; s < AS; s++) sVal[s * vmax + v] = __fmul_rn(vals[s], G.delta_t);
      }
    }
    int ne = 0;
    if (AMODE != 0 && !skip_all) {
      long long s0;
      float sc;
      if (PF) {
        s0 = sMeta[mb].s0;
        ne = (int)(sMeta[mb].s1 - s0);
        sc = sMeta[mb].sc;
      } else {
        const long long ti = (long long)fr * A.n_masked + A.col_rank[row * G.N_x + col];
        s0 = A.tstart[ti];
        ne = (int)(A.tstart[ti + 1] - s0);
        sc = (AMODE == 1) ? A.tscale[ti] : 1.f;
      }
      if (!PFE) {
        for (int e = tid; e < ne; e += NT) {
          const float a = (AMODE == 2) ? __ldg(A.tval32 + s0 + e) : __half2float(A.tval16[s0 + e]) * sc;
          sEnt[e] = make_int2(__ldg(A.toff + s0 + e), __float_as_int(a));
        }
      }
    }
    if (PFE) cp_wait_all();
    __syncthreads();
    // The next item's chain steps are issued by thread 0 where a phase of
    // this item follows that needs none of its own asynchronous copies (its
    // waits complete every copy it has in flight): the rank during the
    // footprint loop, the run bounds during the surrogate step.
    if (PF && tid == 0) {
      cp_wait_all();  // the next item's record
      fetch_rank();
    }

    // 3. theta1 / theta2 over the column's footprint (XT_VoxUpdate.c:20-51)
    const int tln = (T + VEC - 1) / VEC;
    // threads per entry tlp = 2^lg >= tln; the small CTAs group by shifts
    // (+3 % on 16-row items), the 256-thread ones keep the division (0.5 %
    // faster there as measured)
    int lg = 0;
    while ((1 << lg) < tln) lg++;
    const int tlp = 1 << lg;
    const int vgs = NT < XTG_THREADS ? NT >> lg : NT / tlp, tl = tid & (tlp - 1),
              vg = NT < XTG_THREADS ? tid >> lg : tid / tlp;
    float th1[VEC], th2[VEC];
#pragma unroll
    for (int c = 0; c < VEC; c++) th1[c] = th2[c] = 0.f;
    // one footprint entry: rows [off, off + VEC) past this thread's first row
    // of one (view, bin), weight a.  Generalized-Huber (zinger) weight
    // (XT_VoxUpdate.c:34-48): w where |e sqrt(w)| < T, else
    // we = T delta sqrt(w) / |e| = T delta w rsqrt(e^2 w), so that
    //   theta2 += a^2 we = a^2 T delta sqrt(w) / |e|,
    //   theta1 -= a e we = a T delta sign(e) sqrt(w);
    // rsqrt comes from the special-function unit, and the weighted branch
    // runs only when some lane of the warp meets a zinger.
    const int trow0 = t0 + tl * VEC;
    const float *eb = A.e + trow0;
    const float *wb = A.w + trow0;
    auto accumulate_arr = [&](const float (&ev)[VEC], const float (&wv)[VEC], float a) {
      const float a2 = a * a, na = -a;
      if constexpr (VEC == 4 && XTG_F32X2) {
        // two rows per instruction on the packed FP32 path; every product and
        // fused multiply-add is rounded as the scalar one would be
        const float2 e0 = make_float2(ev[0], ev[1]), e1 = make_float2(ev[2], ev[3]);
        const float2 w0 = make_float2(wv[0], wv[1]), w1 = make_float2(wv[2], wv[3]);
        const float2 ew0 = __fmul2_rn(e0, w0), ew1 = __fmul2_rn(e1, w1);
        const float2 q0 = __fmul2_rn(e0, ew0), q1 = __fmul2_rn(e1, ew1);  // e^2 w
        const float qm = fmaxf(fmaxf(q0.x, q0.y), fmaxf(q1.x, q1.y));
        const float2 aa = make_float2(a2, a2), nn = make_float2(na, na);
        float2 t20 = make_float2(th2[0], th2[1]), t21 = make_float2(th2[2], th2[3]);
        float2 t10 = make_float2(th1[0], th1[1]), t11 = make_float2(th1[2], th1[3]);
        if (__any_sync(__activemask(), qm >= A.T2)) {
          // the weight is w, or T delta w / sqrt(e^2 w) (= T delta sqrt(w) / |e|)
          // where |e sqrt(w)| >= T
          auto wgt = [&](float q, float w) { return q >= A.T2 ? A.Tdelta * w * rsqrtf(q) : w; };
          const float2 we0 = make_float2(wgt(q0.x, w0.x), wgt(q0.y, w0.y));
          const float2 we1 = make_float2(wgt(q1.x, w1.x), wgt(q1.y, w1.y));
          t20 = __ffma2_rn(aa, we0, t20);
          t21 = __ffma2_rn(aa, we1, t21);
          t10 = __ffma2_rn(nn, __fmul2_rn(e0, we0), t10);
          t11 = __ffma2_rn(nn, __fmul2_rn(e1, we1), t11);
        } else {
          t20 = __ffma2_rn(aa, w0, t20);
          t21 = __ffma2_rn(aa, w1, t21);
          t10 = __ffma2_rn(nn, ew0, t10);
          t11 = __ffma2_rn(nn, ew1, t11);
        }
        th2[0] = t20.x; th2[1] = t20.y; th2[2] = t21.x; th2[3] = t21.y;
        th1[0] = t10.x; th1[1] = t10.y; th1[2] = t11.x; th1[3] = t11.y;
        return;
      }
      float ew[VEC], q[VEC];
      float qm = 0.f;
#pragma unroll
      for (int c = 0; c < VEC; c++) {
        ew[c] = ev[c] * wv[c];
        q[c] = ev[c] * ew[c];  // e^2 w
        qm = fmaxf(qm, q[c]);
      }
      if (__any_sync(__activemask(), qm >= A.T2)) {
        // branch-free per row: the weight is w, or T delta w / sqrt(e^2 w)
        // (= T delta sqrt(w) / |e|) where |e sqrt(w)| >= T
#pragma unroll
        for (int c = 0; c < VEC; c++) {
          const float we = q[c] >= A.T2 ? A.Tdelta * wv[c] * rsqrtf(q[c]) : wv[c];
          th2[c] = fmaf(a2, we, th2[c]);
          th1[c] = fmaf(na, ev[c] * we, th1[c]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < VEC; c++) {
          th2[c] = fmaf(a2, wv[c], th2[c]);
          th1[c] = fmaf(na, ew[c], th1[c]);
        }
      }
    };
    auto accumulate_vals = [&](const float4 e4, const float4 w4, float a) {
      float ev[VEC], wv[VEC];
      const float ea[4] = {e4.x, e4.y, e4.z, e4.w}, wa[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int c = 0; c < VEC; c++) {
        ev[c] = ea[c < 4 ? c : 0];
        wv[c] = wa[c < 4 ? c : 0];
      }
      accumulate_arr(ev, wv, a);
    };
    auto accumulate = [&](int off, float a) {
      float ev[VEC], wv[VEC];
      if (VEC == 4) {
        const float4 e4 = ld_e(eb + off);
        const float4 w4 = ld_w(wb + off, A.w_keep);
        ev[0] = e4.x; ev[1] = e4.y; ev[2] = e4.z; ev[3] = e4.w;
        wv[0] = w4.x; wv[1] = w4.y; wv[2] = w4.z; wv[3] = w4.w;
      } else {
#pragma unroll
        for (int c = 0; c < VEC; c++) {
          ev[c] = __ldcg(eb + off + c);
          wv[c] = __ldg(wb + off + c);
        }
      }
      accumulate_arr(ev, wv, a);
    };
    if (tl < tln && !skip_all) {
      if (AMODE == 0) {
        for (int v = vg; v < V; v += vgs) {
          const int pk = sPack[v], first = pk & 0xffffff, n = pk >> 24;
          const int off = (sView[v] * G.N_r + first) * G.N_t;
#pragma unroll
          for (int s = 0; s < AS; s++)
            if (s < n) accumulate(off + s * G.N_t, sVal[s * vmax + v]);
        }
      } else if (VEC == 4) {
        int e = vg;
        constexpr int UNR = NT < XTG_THREADS ? 2 : XTG_UNROLL;
        for (; e + (UNR - 1) * vgs < ne; e += UNR * vgs) {
          int2 en[UNR];
          float4 e4[UNR], w4[UNR];
#pragma unroll
          for (int u = 0; u < UNR; u++) en[u] = sEnt[e + u * vgs];
#pragma unroll
          for (int u = 0; u < UNR; u++) {
            e4[u] = ld_e(eb + en[u].x);
            w4[u] = ld_w(wb + en[u].x, A.w_keep);
          }
#pragma unroll
          for (int u = 0; u < UNR; u++) accumulate_vals(e4[u], w4[u], __int_as_float(en[u].y));
        }
        for (; e < ne; e += vgs) {
          const int2 en = sEnt[e];
          accumulate(en.x, __int_as_float(en.y));
        }
      } else {
        for (int e = vg; e < ne; e += vgs) {
          const int2 en = sEnt[e];
          accumulate(en.x, __int_as_float(en.y));
        }
      }
    }
    // reduce over view groups: lanes with equal tl inside a warp, then warps
#pragma unroll
    for (int c = 0; c < VEC; c++) {
      for (int off = tlp; off < 32; off <<= 1) {
        th1[c] += __shfl_xor_sync(0xffffffffu, th1[c], off);
        th2[c] += __shfl_xor_sync(0xffffffffu, th2[c], off);
      }
    }
    if (lane < tlp && tl < tln) {
#pragma unroll
      for (int c = 0; c < VEC; c++) {
        sRed[warp * 128 + tl * VEC + c] = th1[c];
        sRed[NW * 128 + warp * 128 + tl * VEC + c] = th2[c];
      }
    }
    __syncthreads();
    if (PF && tid == 0) {
      cp_wait_all();
      fetch_bounds();
    }
    for (int t = tid; t < T; t += NT) {
      float s1 = 0.f, s2 = 0.f;
#pragma unroll
      for (int wq = 0; wq < NW; wq++) {  // every warp wrote its partial (zeros if idle)
        s1 += sRed[wq * 128 + t];
        s2 += sRed[NW * 128 + wq * 128 + t];
      }
      sTh[t] = s1;
      sTh[rowsmax + t] = s2;
    }
    __syncthreads();

    // 4. qGGMRF surrogate step per slice (CE_FunctionalSubstitution,
    //    XT_ICD_update.c:130-179) with zero skipping (XT_VoxUpdate.c:208-232)
    double absx = 0.0;
    if (SEQ) {
      if (tid == 0) {
        for (int z = 0; z < Z; z++) {
          const float Vv = sNb[4 * (zmax + 2) + z + 1];
          float t1 = 0.f, t2 = 0.f;
          for (int r = 0; r < G.zovl; r++) {
            t1 += sTh[z * G.zovl + r];
            t2 += sTh[rowsmax + z * G.zovl + r];
          }
          bool skip = false;
          if (Vv == 0.f && A.iter > 1) {
            skip = !(sTn[z] > 0.f || sTn[zmax + z] > 0.f);
            for (int c = 0; c < 9 && skip; c++)
              for (int dz = 0; dz < 3; dz++)
                if (sNb[c * (zmax + 2) + z + dz] > 0.f) skip = false;
          }
          if (skip) {
            sDelta[z] = 0.f;
            sZero++;
            continue;
          }
          float num = 0.f, den = 0.f;
          for (int n = 0; n < 29; n++) {
            const Nbr o = nbr_term(G, sNb, sTn, zmax, z, zb, fr, row, col, Vv, n, hlo, hhi);
            num += o.b * o.v;
            den += o.b;
          }
          const float u = (num + t2 * Vv - t1) / (den + t2);
          float nvx = Vv + G.alpha * (u - Vv);
          if (G.positivity && nvx <= 0.f) nvx = 0.f;
          if (!isfinite(nvx)) {
            atomicExch(A.err, 1);
            nvx = Vv;
          }
          sNb[4 * (zmax + 2) + z + 1] = nvx;
          A.x[(((size_t)fr * plane) + (size_t)row * G.N_x + col) * G.N_z + zb + z] = nvx;
          sDelta[z] = nvx - Vv;
          absx += (double)fabsf(nvx);
          sUpd++;
        }
      }
    } else {
      // red/black in z, 8 lanes per voxel, each lane a subset of the 29
      // neighbour slots; the lane group reduces with shuffles
      const int sub = tid & 7, slot = tid >> 3;
      for (int par = 0; par < 2; par++) {
        const int zfirst = ((zb & 1) == par) ? 0 : 1;  // first z (relative) with absolute parity par
        const int nvox = (Z - zfirst + 1) / 2;
        for (int s0 = 0; s0 < nvox; s0 += NT / 8) {
          const int vi = s0 + slot;
          const bool act = vi < nvox;
          const int z = zfirst + 2 * (act ? vi : 0);
          const float Vv = sNb[4 * (zmax + 2) + z + 1];
          // zero skipping: V == 0 from the second iteration and no positive neighbour
          bool pos = false;
          float num = 0.f, den = 0.f;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int n = sub + 8 * k;
            if (n < 29) {
              const Nbr o = nbr_term(G, sNb, sTn, zmax, z, zb, fr, row, col, Vv, n, hlo, hhi);
              num += o.b * o.v;
              den += o.b;
            }
          }
          // positive-neighbour test over the raw values (absent slots read 0)
          if (Vv == 0.f && A.iter > 1) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const int n = sub + 8 * k;
              if (n < 27) {
                if (sNb[(n % 9) * (zmax + 2) + z + n / 9] > 0.f) pos = true;
              } else if (n < 29) {
                if (sTn[(n - 27) * zmax + z] > 0.f) pos = true;
              }
            }
          }
#pragma unroll
          for (int off = 1; off < 8; off <<= 1) {
            num += __shfl_xor_sync(0xffffffffu, num, off);
            den += __shfl_xor_sync(0xffffffffu, den, off);
            pos |= __shfl_xor_sync(0xffffffffu, (int)pos, off) != 0;
          }
          if (act && sub == 0) {
            const int zr = z;
            if (Vv == 0.f && A.iter > 1 && !pos) {
              sDelta[zr] = 0.f;
              atomicAdd(&sZero, 1u);
            } else {
              float t1 = 0.f, t2 = 0.f;
              for (int r = 0; r < G.zovl; r++) {
                t1 += sTh[zr * G.zovl + r];
                t2 += sTh[rowsmax + zr * G.zovl + r];
              }
              const float u = (num + t2 * Vv - t1) / (den + t2);
              float nvx = Vv + G.alpha * (u - Vv);
              if (G.positivity && nvx <= 0.f) nvx = 0.f;
              if (!isfinite(nvx)) {
                atomicExch(A.err, 1);
                nvx = Vv;
              }
              sNb[4 * (zmax + 2) + zr + 1] = nvx;
              A.x[(((size_t)fr * plane) + (size_t)row * G.N_x + col) * G.N_z + zb + zr] = nvx;
              sDelta[zr] = nvx - Vv;
              absx += (double)fabsf(nvx);
              atomicAdd(&sUpd, 1u);
            }
          }
        }
        __syncthreads();
      }
    }
    __syncthreads();

    // 5. MagUpdateMap[frame][block][row][col] = sum |delta| over the block's
    //    slices of this visit (XT_VoxUpdate.c:128, 236); sum |x| and counters
    for (int b = tid; b < G.nzb; b += NT) {
      const int bz0 = b * G.zstep, bz1 = (b >= G.nzb - 1) ? G.N_z - 1 : (b + 1) * G.zstep - 1;
      const int lo = max(bz0, zb), hi = min(bz1, ze);
      float *mp = A.magmap + (((size_t)fr * G.nzb + b) * G.N_y + row) * G.N_x + col;
      if (A.nsub > 1) {
        // pieces of one block add into the entry zeroed before the launch
        if (lo <= hi) {
          float m = 0.f;
          for (int z = lo; z <= hi; z++) m += fabsf(sDelta[z - zb]);
          atomicAdd(mp, m);
        }
      } else if (bz0 >= zb && bz1 <= ze) {
        float m = 0.f;
        for (int z = bz0; z <= bz1; z++) m += fabsf(sDelta[z - zb]);
        *mp = m;
      }
    }
    for (int off = 16; off > 0; off >>= 1) absx += __shfl_xor_sync(0xffffffffu, absx, off);
    if (lane == 0) sAbs[warp] = absx;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int wq = 0; wq < NT / 32; wq++) s += sAbs[wq];
      sCtaAbs += s;
      sCta[0] += sUpd;
      sCta[1] += sZero;
      if (piece == 0) sCta[2]++;
    }

    // 6. e -= (A delta_t) * delta_x on the footprint (XT_VoxUpdate.c:62-82)
    if (tl < tln) {
      float dv[VEC];
      bool any = false;
#pragma unroll
      for (int c = 0; c < VEC; c++) {
        const int rr = tl * VEC + c;
        dv[c] = (rr < T) ? sDelta[G.zovl == 1 ? rr : rr / G.zovl] : 0.f;
        any |= (dv[c] != 0.f);
      }
      if (any) {
        float *ebw = A.e + trow0;
        auto scatter = [&](int off, float a) {
          if constexpr (VEC == 4 && XTG_F32X2) {
            const float2 na2 = make_float2(-a, -a);
            const float2 m0 = __fmul2_rn(na2, make_float2(dv[0], dv[1]));
            const float2 m1 = __fmul2_rn(na2, make_float2(dv[2], dv[3]));
            xt_red_add4(ebw + off, m0.x, m0.y, m1.x, m1.y);
          } else if (VEC == 4) {
            xt_red_add4(ebw + off, -(a * dv[0]), -(a * dv[1]), -(a * dv[2]), -(a * dv[3]));
          } else {
#pragma unroll
            for (int c = 0; c < VEC; c++)
              if (dv[c] != 0.f) atomicAdd(ebw + off + c, -(a * dv[c]));
          }
        };
        if (AMODE == 0) {
          for (int v = vg; v < V; v += vgs) {
            const int pk = sPack[v], first = pk & 0xffffff, n = pk >> 24;
            const int off = (sView[v] * G.N_r + first) * G.N_t;
#pragma unroll
            for (int s = 0; s < AS; s++)
              if (s < n) scatter(off + s * G.N_t, sVal[s * vmax + v]);
          }
        } else {
          for (int e = vg; e < ne; e += vgs) {
            const int2 en = sEnt[e];
            scatter(en.x, __int_as_float(en.y));
          }
        }
      }
    }
    if (PF && tid == 0) cp_wait_all();  // the next item's meta is complete
    __syncthreads();
    mb ^= 1;
  }
  if (tid == 0 && (sCta[0] || sCta[1] || sCta[2] || sCtaAbs != 0.0)) {  // pieces past the first count no item
    atomicAdd(&A.st_absx[blockIdx.x & 63], sCtaAbs);
    atomicAdd(&A.st_cnt[0], sCta[0]);
    atomicAdd(&A.st_cnt[1], sCta[1]);
    atomicAdd(&A.st_cnt[2], sCta[2]);
  }
}

size_t icd_smem_bytes(int vmax, int zmax, int zovl, int as, int amode, int vec, int nt) {
  size_t b = 0;
  if (amode == 0)
    b += (size_t)vmax * (4 * 2 + 4 * (size_t)as);  // sPack, sView, sVal
  else
    b += (size_t)vmax * 8;                         // sEnt
  b += 2 * (size_t)(nt / 32) * 128 * 4;            // sRed
  b += 2 * (size_t)zmax * zovl * 4;                // sTh
  b += 9 * (size_t)(zmax + 2) * 4;                 // sNb
  b += 2 * (size_t)zmax * 4;                       // sTn
  b += (size_t)zmax * 4;                           // sDelta
  return b;
}


typedef void (*IcdKernel)(DevGeo, IcdArgs, int, int);

// A computed in the kernel (amode 0): slot count 3 covers delta_xy <= delta_r,
// 4 covers delta_xy <= 1.5 delta_r, 12 covers delta_xy <= 5.5 delta_r.  The
// table modes (1 = FP16, 2 = FP32) have no per-view slots.
static IcdKernel icd_kernel(int vec, int amode, int seq, int as, int nt) {
#define XTG_K(V, S) (as == 3 ? k_icd_columns<V, 0, S, 3> : as == 4 ? k_icd_columns<V, 0, S, 4> : k_icd_columns<V, 0, S, 12>)
#define XTG_T(V, M, S) k_icd_columns<V, M, S, 3>
  if (nt != XTG_THREADS && vec == 4 && amode != 0 && !seq)  // short items, table modes
    return nt == XTG_SMALL_NT ? (amode == 1 ? k_icd_columns<4, 1, 0, 3, XTG_SMALL_NT> : k_icd_columns<4, 2, 0, 3, XTG_SMALL_NT>)
                              : (amode == 1 ? k_icd_columns<4, 1, 0, 3, XTG_MEDIUM_NT> : k_icd_columns<4, 2, 0, 3, XTG_MEDIUM_NT>);
  if (vec == 4) {
    if (amode == 0) return seq ? XTG_K(4, 1) : XTG_K(4, 0);
    if (amode == 1) return seq ? XTG_T(4, 1, 1) : XTG_T(4, 1, 0);
    return seq ? XTG_T(4, 2, 1) : XTG_T(4, 2, 0);
  }
  if (amode == 0) return seq ? XTG_K(1, 1) : XTG_K(1, 0);
  if (amode == 1) return seq ? XTG_T(1, 1, 1) : XTG_T(1, 1, 0);
  return seq ? XTG_T(1, 2, 1) : XTG_T(1, 2, 0);
#undef XTG_K
#undef XTG_T
}

// Zeroes MagUpdateMap[frame][block][row][col] for every (item, block the
// item covers) of an ICD launch whose items are split into z pieces, which
// then add their partial sums into it.
__global__ void k_magmap_zero(DevGeo G, IcdArgs A) {
  const int nitems = A.n_items_dev ? *A.n_items_dev : A.n_items;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nitems; i += gridDim.x * blockDim.x) {
    const int q = A.use_perm ? (int)xt_perm((uint32_t)i, (uint32_t)nitems, A.perm_key) : i;
    const int4 item = A.items[A.item_lo + q];
    const int b0 = item.w >= 0 ? item.w : 0, b1 = item.w >= 0 ? item.w : G.nzb - 1;
    for (int b = b0; b <= b1; b++)
      A.magmap[(((size_t)item.x * G.nzb + b) * G.N_y + item.y) * G.N_x + item.z] = 0.f;
  }
}

cudaError_t launch_magmap_zero(const DevGeo &G, const IcdArgs &A, int grid, cudaStream_t st) {
  k_magmap_zero<<<grid, 256, 0, st>>>(G, A);
  return cudaGetLastError();
}

// threads per CTA for items of zmax slices: XTG_SMALL_NT for short table-mode items
int icd_threads(int vec, int amode, int seq, int zmax, int zovl, int vmax) {
  if (vec == 4 && amode != 0 && !seq && zmax * zovl <= XTG_SMALL_ROWS) return XTG_SMALL_NT;
  if (vec == 4 && amode != 0 && !seq && vmax <= XTG_MEDIUM_ENTRIES) return XTG_MEDIUM_NT;
  return XTG_THREADS;
}

cudaError_t launch_icd(const DevGeo &G, const IcdArgs &A, int vec, int amode, int seq, int as, int vmax, int zmax,
                       int grid, cudaStream_t st) {
  const int nt = icd_threads(vec, amode, seq, zmax, G.zovl, vmax);
  const size_t smem = icd_smem_bytes(vmax, zmax, G.zovl, as, amode, vec, nt);
  IcdKernel k = icd_kernel(vec, amode, seq, as, nt);
  cudaError_t e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // e and w stream through L2 (e must, it is updated by other CTAs' atomics),
  // so give the unified L1/shared space to shared memory: more CTAs per SM
  e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  k<<<grid, nt, smem, st>>>(G, A, vmax, zmax);
  return cudaGetLastError();
}

int icd_occupancy(int vec, int amode, int seq, int as, int vmax, int zmax, int zovl) {
  const int nt = icd_threads(vec, amode, seq, zmax, zovl, vmax);
  const size_t smem = icd_smem_bytes(vmax, zmax, zovl, as, amode, vec, nt);
  IcdKernel k = icd_kernel(vec, amode, seq, as, nt);
  int nb = 0;
  cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute((const void *)k, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)k, nt, smem) != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

}  // namespace xtg
