// tile_search.cu -- the BF16+refine form of the join's search: tensor-core
// (tcgen05) distance tiles with rigorous error bounds, exact FP32 re-ranking
// and an FP64 re-check of the k-th boundary.
//
// It replaces the per-query scan (KNNQuery_base, src/knnjoin.cu:762-858) for
// the same clusters, bounds and candidate cluster lists: the reference
// computes every surviving distance in FP32 on CUDA cores; here a CTA takes
// a tile of up to 128 queries of one query cluster and streams the members
// of that cluster's candidate list (nearest cluster first) through a
// 128 x 128 x KD BF16 MMA with FP32 accumulation in TMEM:
//   - rows are centred on one query point of the cluster before rounding to
//     BF16, so the rounded values (and their errors) are small; data on an
//     integer grid stays exact;
//   - for every (query, member) pair the epilogue turns the dot product into
//     a lower bound L and an upper bound U of the exact squared distance,
//         L, U = |a|^2 + |b|^2 -/+ slack - 2 acc -/+ delta,
//     where delta bounds the BF16 rounding (|a| |b - b~| + |a - a~| |b~|)
//     and the tensor-core accumulation, from per-row norms computed in FP32;
//   - each query keeps, in a global-memory buffer, every pair whose L is at
//     most the k-th smallest U seen so far (initially theta0^2, the cluster's
//     k-th distance bound): no pair outside can be among the k nearest.
//     When a buffer fills, a warp selects the k-th U (radix select) and
//     compacts it;
//   - at the end a warp per query recomputes the kept pairs exactly in FP32
//     (the same arithmetic as the FP32 scan), selects the k smallest keys
//     (d^2, index), and re-decides every key within the FP32 rounding band of
//     the k-th in FP64 (ties to the lower index).  The neighbour set is
//     therefore the one an FP64 join gives.
// A query whose buffer cannot hold its kept pairs (for example thousands of
// duplicate points at the boundary) is handed to the FP32 scan.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_common.cuh"
#include "warp_select.cuh"

namespace knnsweet {

namespace {

// Optional phase timers (build with -DKNN_TILE_PROFILE=1): thread 0 of every
// CTA adds the clock cycles between its barriers to tile_prof[phase].
// Clusters in the first batch (they tighten the bounds before the rest of the
// list is decided) and the growth of a row's compaction limit after a
// compaction (GROW / 2 times the kept pairs, plus 32).
#ifndef KNN_TILE_FIRST
#define KNN_TILE_FIRST 4
#endif
// (first batch 2 / 4 / 8: C3 search 10.5 / 11.1 / 11.2 ms, C2 11.9 / 4.2 /
// 4.6 ms; growth 3 / 4 / 6: C2 4.29 / 4.24 / 4.13-4.16 ms, C3 unchanged)
#ifndef KNN_TILE_GROW
#define KNN_TILE_GROW 6
#endif
#ifndef KNN_TILE_PROFILE
#define KNN_TILE_PROFILE 0
#endif
#if KNN_TILE_PROFILE
__device__ unsigned long long tile_prof[16];
#define TILE_PROF(i)                                  \
  do {                                                \
    if (tid == 0) {                                   \
      const long long now_ = clock64();               \
      prof[i] += (unsigned long long)(now_ - prof_t); \
      prof_t = now_;                                  \
    }                                                 \
  } while (0)
#else
#define TILE_PROF(i) \
  do {               \
  } while (0)
#endif

constexpr int kTM = 128;  // queries per tile: TMEM lanes, the row threads of a CTA
constexpr int kTN = 128;  // member rows per chunk: TMEM columns
// Threads per CTA (template NT): the first kTM own the tile's rows (TMEM
// lanes) through the epilogue.  With NT = 2 kTM all of them stage tiles and
// share out the re-ranking, so that the latency-bound CTA keeps twice the
// warps in flight at the same shared memory; that pays where the re-ranking
// state of four more warps fits the tile region (wide rows, d = 128: C3
// search 16.0 -> 13.2 ms).  Otherwise NT = kTM keeps four CTAs per SM.

// Tile list: every query cluster's slots in tiles of up to kTM, as
// {query cluster, first slot, count, slot of the cluster's centre point}.
// The centre is the cluster's first slot: the query nearest its
// representative.  One block of 1024 threads, each owning a run of clusters.
__global__ void __launch_bounds__(1024)
    tile_list_kernel(const int32_t *__restrict__ qoff, int Rq, int c_base,
                     int32_t *__restrict__ tiles, int32_t *__restrict__ ntiles) {
  __shared__ int wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (Rq + 1023) / 1024;
  const int c0 = min(Rq, tid * per), c1 = min(Rq, c0 + per);
  int local = 0;
  for (int c = c0; c < c1; c++) local += (qoff[c + 1] - qoff[c] + kTM - 1) / kTM;
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int v = wsum[lane];
    int iv = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, iv, o);
      if (lane >= o) iv += t;
    }
    wsum[lane] = iv - v;
  }
  __syncthreads();
  int pos = wsum[warp] + incl - local;
  for (int c = c0; c < c1; c++) {
    const int size = qoff[c + 1] - qoff[c];
    for (int s = 0; s < size; s += kTM) {
      tiles[4 * pos + 0] = c_base + c;
      tiles[4 * pos + 1] = qoff[c] + s;
      tiles[4 * pos + 2] = min(kTM, size - s);
      tiles[4 * pos + 3] = qoff[c];
      pos++;
    }
  }
  if (tid == 1023) *ntiles = pos;
}

// Rows r of a 128-row tile, centred on sc, rounded to BF16 into the
// core-matrix layout of tc_common.cuh; per row the sums
//   o_n = sum v^2, o_e = sum (v - bf16(v))^2, o_t = sum bf16(v)^2
// of the centred FP32 values v.  rowptr(r) gives the row (nullptr: zeros).
// G = KD/8 consecutive threads share a row (one 16-byte group each).
template <int NT, class RowPtr>
__device__ __forceinline__ void stage_tile(unsigned char *tile, const float *sc, int KD, int d,
                                           int dp4, RowPtr rowptr, float *o_n, float *o_e,
                                           float *o_t) {
  const int G = KD >> 3;
  // four 16-byte groups per thread per round, their loads issued together
  // (whether a round's group exists depends only on the round: uniform)
  for (int t0 = threadIdx.x; t0 < kTM * G; t0 += 4 * NT) {
    float4 c0[4], c1[4];
    bool has[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int t = t0 + u * NT;
      const int r = t / G, k0 = (t - r * G) << 3;
      const float4 *row = t < kTM * G ? rowptr(r) : nullptr;
      has[u] = row != nullptr;
      c0[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      c1[u] = c0[u];
      if (row) {
        if ((k0 >> 2) < dp4) c0[u] = row[k0 >> 2];
        if ((k0 >> 2) + 1 < dp4) c1[u] = row[(k0 >> 2) + 1];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int t = t0 + u * NT;
      if (t >= kTM * G) break;
      const int r = t / G, g = t - r * G, k0 = g << 3;
      const float v[8] = {c0[u].x, c0[u].y, c0[u].z, c0[u].w,
                          c1[u].x, c1[u].y, c1[u].z, c1[u].w};
      float sn = 0.0f, se = 0.0f, st = 0.0f;
      __align__(16) __nv_bfloat16 h[8];
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int kk = k0 + e;
        const float x = (has[u] && kk < d) ? __fsub_rn(v[e], sc[kk]) : 0.0f;
        h[e] = __float2bfloat16_rn(x);
        const float xr = __bfloat162float(h[e]);
        const float df = __fsub_rn(x, xr);
        sn = __fmaf_rn(x, x, sn);
        se = __fmaf_rn(df, df, se);
        st = __fmaf_rn(xr, xr, st);
      }
      *reinterpret_cast<uint4 *>(tile + tc::tile_offset(r, k0, KD)) =
          *reinterpret_cast<const uint4 *>(h);
      for (int o = G >> 1; o > 0; o >>= 1) {
        sn += __shfl_xor_sync(kFull, sn, o);
        se += __shfl_xor_sync(kFull, se, o);
        st += __shfl_xor_sync(kFull, st, o);
      }
      if (g == 0) {
        o_n[r] = sn;
        o_e[r] = se;
        o_t[r] = st;
      }
    }
  }
}

// Keeps the entries of a bound buffer (lu, pos: n entries in shared memory)
// whose lower bound is at most the k-th smallest upper bound, or an upper
// bound of it -- no entry beyond it can be among the k nearest; in place, by
// one warp.  Returns the count kept and that bound.  Needs n >= k.
__device__ __forceinline__ int compact_bounds(float2 *lu, int32_t *pos, int n, int k,
                                              uint32_t *hist, int lane, float *uk_out) {
#if KNN_LINEAR_SELECT
  const float uk = __uint_as_float(
      warp_kth_upper_u32(reinterpret_cast<const uint32_t *>(lu) + 1, 2, n, k, hist, lane));
#else
  const float uk = __uint_as_float(
      warp_select_kth_u32(reinterpret_cast<const uint32_t *>(lu) + 1, 2, n, k, hist, lane));
#endif
  int w = 0;
  for (int b0 = 0; b0 < n; b0 += 32) {
    const int i = b0 + lane;
    float2 v = make_float2(0.0f, 0.0f);
    int32_t p = 0;
    if (i < n) {
      v = lu[i];
      p = pos[i];
    }
    const bool keep = i < n && v.x <= uk;
    const unsigned bm = __ballot_sync(kFull, keep);
    if (keep) {
      const int o = w + __popc(bm & ((1u << lane) - 1u));
      lu[o] = v;
      pos[o] = p;
    }
    w += __popc(bm);
  }
  __syncwarp();
  *uk_out = uk;
  return w;
}

// Copies n buffer entries between global and shared memory, by one warp.
__device__ __forceinline__ void copy_entries(float2 *dlu, int32_t *dpos, const float2 *slu,
                                             const int32_t *spos, int n, int lane) {
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    dlu[i] = slu[i];
    dpos[i] = spos[i];
  }
  __syncwarp();
}

// Exact squared distance in FP32 over the first d columns, in column order:
// the value the FP32 scan computes for the same pair (padding columns add
// exact zeros there).  Rows are float4-aligned.
__device__ __forceinline__ float dist2_cols(const float4 *__restrict__ q,
                                            const float4 *__restrict__ r, int d) {
  float acc = 0.0f;
  const int full = d >> 2;
  for (int c = 0; c < full; c++) {
    const float4 u = q[c], v = r[c];
    float t;
    t = __fsub_rn(u.x, v.x); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.y, v.y); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.z, v.z); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.w, v.w); acc = __fmaf_rn(t, t, acc);
  }
  const int rem = d & 3;
  if (rem) {
    const float4 u = q[full], v = r[full];
    float t;
    t = __fsub_rn(u.x, v.x); acc = __fmaf_rn(t, t, acc);
    if (rem > 1) { t = __fsub_rn(u.y, v.y); acc = __fmaf_rn(t, t, acc); }
    if (rem > 2) { t = __fsub_rn(u.z, v.z); acc = __fmaf_rn(t, t, acc); }
  }
  return acc;
}

// Sorts the n <= 32E keys s[0..n) ascending in registers (padding with the
// largest key) and writes 32E sorted keys back to s.  One warp.
template <int E>
__device__ __forceinline__ void sort_keys_in_registers(uint64_t *s, int n, int lane) {
  uint64_t x[E];
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int p = j * 32 + lane;
    x[j] = p < n ? s[p] : kKeyMax;
  }
  __syncwarp();
  reg_bitonic_sort<E>(x, lane);
#pragma unroll
  for (int j = 0; j < E; j++) s[E * lane + j] = x[j];
  __syncwarp();
}

// Bytes of the query and member tiles at the start of shared memory.
__host__ __device__ constexpr size_t tiles_bytes(int KD) {
  return tc::tile_bytes(kTM, KD) + tc::tile_bytes(kTN, KD);
}

template <int NT>
__global__ void __launch_bounds__(NT, NT == kTM ? 4 : 2)
    tile_search_kernel(const TileArgs a) {
  constexpr int kThreads = NT, kWarps = NT / 32;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int KD = a.KD, d = a.d, dp4 = a.dp4, k = a.k, cap = a.cap, P = a.P;
  (void)P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *sa = smem;                                      // kTM x KD bf16
  unsigned char *sb = sa + tc::tile_bytes(kTM, KD);              // kTN x KD bf16
  float *sc = reinterpret_cast<float *>(sb + tc::tile_bytes(kTN, KD));  // KD
  float4 *s_col = reinterpret_cast<float4 *>(sc + KD);          // kTN column scalars
  float *s_n = reinterpret_cast<float *>(s_col + kTN);           // kTN row sums
  float *s_e = s_n + kTN;
  float *s_t = s_e + kTN;
  int32_t *s_pos = reinterpret_cast<int32_t *>(s_t + kTN);      // kTN member positions
  int32_t *s_rlo = s_pos + kTN;                                  // kTN run starts
  int32_t *s_roff = s_rlo + kTN;                                 // kTN run offsets
  float *s_cmin = reinterpret_cast<float *>(s_roff + kTN);       // kTN per batch cluster
  float *s_cmax = s_cmin + kTN;
  float *s_ck = s_cmax + kTN;                                    // k-th member distance
  uint32_t *s_blo = reinterpret_cast<uint32_t *>(s_ck + kTN);    // run bounds (float bits)
  uint32_t *s_bhi = s_blo + kTN;
  int32_t *s_wsum = reinterpret_cast<int32_t *>(s_bhi + kTN);    // kWarps warp sums
  uint32_t *s_wmax = reinterpret_cast<uint32_t *>(s_wsum + kWarps);  // [1]: run total
  uint32_t *hist = s_wmax + 4;                                   // 4 x 256
  uint64_t *mbar = reinterpret_cast<uint64_t *>(hist + 4 * 256);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);
  int32_t *s_tile = reinterpret_cast<int32_t *>(tmem_slot + 1);  // 4 ints
  // warps 0-3: one query's buffer each (cap bound pairs, cap positions), a
  // query row and a histogram, for the compactions between member chunks
  // and the final re-ranking; warps 4-7 join the re-ranking only, once the
  // tiles are no longer needed, with the same state inside the tile region
  const size_t wofs = ((size_t)(reinterpret_cast<unsigned char *>(s_tile + 4) - smem) + 15) &
                      ~(size_t)15;
  const size_t wstate = (size_t)cap * 12 + (size_t)dp4 * 16 + 256 * 4;  // bytes per warp
  const bool rerank_all = kWarps > 4 && 4 * wstate <= tiles_bytes(KD);
  float4 *wq;
  unsigned char *wbase;
  uint32_t *whist;
  if (warp < 4) {
    wq = reinterpret_cast<float4 *>(smem + wofs) + (size_t)warp * dp4;
    wbase = smem + wofs + 4 * (size_t)dp4 * 16 + (size_t)warp * cap * 12;
    whist = hist + warp * 256;
  } else {
    unsigned char *w0 = smem + (size_t)(warp - 4) * wstate;
    wbase = w0;
    wq = reinterpret_cast<float4 *>(w0 + (size_t)cap * 12);
    whist = reinterpret_cast<uint32_t *>(w0 + (size_t)cap * 12 + (size_t)dp4 * 16);
  }
  float2 *w_lu = reinterpret_cast<float2 *>(wbase);
  int32_t *w_pos = reinterpret_cast<int32_t *>(wbase + (size_t)cap * 8);
  // warps sharing out the final re-ranking
  const int nrw = rerank_all ? kWarps : 4;

  if (warp == 0) tc::tmem_alloc(tmem_slot, kTN);
  if (tid == 0) tc::mbar_init(mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t idesc = tc::make_idesc_bf16(kTM, kTN);
  const uint32_t a_base = tc::smem_u32(sa), b_base = tc::smem_u32(sb);
  const uint32_t sbo = (uint32_t)KD * 16;
  // relative slack of the FP32 norms, centring and bound arithmetic
  const float kap = (float)(d + 32) * 5.9604645e-8f;
  // tensor-core accumulation error per unit of |a~| |b~|
  const float gtc = (float)(KD + 4) * 2.3841858e-7f;
  // relative slack of the triangle-inequality tests (FP32 rounding of the
  // representative and member distances)
  const float tol = bound_tol(d);
  const size_t row0 = (size_t)blockIdx.x * kTM;
  // this row's global bound buffer (row threads only)
  float2 *my_lu = a.buf_lu + (row0 + (tid & (kTM - 1))) * cap;
  int32_t *my_pos = a.buf_pos + (row0 + (tid & (kTM - 1))) * cap;
  uint32_t phase = 0;
  bool ok = true;
  unsigned long long pairs = 0, refined = 0, rechecks = 0, fallbacks = 0;
#if KNN_TILE_PROFILE
  unsigned long long prof[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long prof_t = clock64();
#endif

  for (;;) {
    if (tid == 0) {
      const unsigned long long w = atomicAdd(a.work, 1ull);
      if (w < (unsigned long long)*a.ntiles) {
#pragma unroll
        for (int i = 0; i < 4; i++) s_tile[i] = a.tiles[4 * w + i];
      } else {
        s_tile[0] = -1;
      }
    }
    __syncthreads();
    const int qc = s_tile[0];
    if (qc < 0) break;
    const int s0 = s_tile[1], cnt = s_tile[2];
    const float *cen = reinterpret_cast<const float *>(a.qrows +
                                                       (size_t)a.qorder[s_tile[3]] * dp4);
    for (int kk = tid; kk < KD; kk += kThreads) sc[kk] = kk < d ? cen[kk] : 0.0f;
    __syncthreads();
    stage_tile<NT>(
        sa, sc, KD, d, dp4,
        [&](int r) -> const float4 * {
          return r < cnt ? a.qrows + (size_t)a.qorder[s0 + r] * dp4 : nullptr;
        },
        s_n, s_e, s_t);
    __syncthreads();
    const bool row_thread = tid < kTM;  // owns tile row (TMEM lane) tid
    const bool valid = tid < cnt;
    const float na = row_thread ? s_n[tid] : 0.0f;
    const float qa = 2.02f * sqrtf(na);
    const float qb = row_thread ? 2.02f * (sqrtf(s_e[tid]) + gtc * sqrtf(s_t[tid])) : 0.0f;
    const float th = a.theta0[qc];
    float tau = th * th * 1.0009765625f;
    // the row's distance to its representative, for the list's early exit
    const float dq_row = valid && a.clb && a.qkeys
                             ? __uint_as_float((uint32_t)a.qkeys[s0 + tid])
                             : __int_as_float(0x7f800000);
    int n = 0;
    bool ovf = false;
    __syncthreads();  // the row sums are reused for the member rows below
    TILE_PROF(0);

    const int32_t *rl = a.rlist + (size_t)qc * a.Rs;
    const int nl = a.rlen[qc];
    int lim = min(cap - kTN, k + 32);  // compact when the buffer passes this
    float th_q = sqrtf(tau);           // this query's k-th distance bound
    // Candidate clusters in batches of 128, nearest first.  One MMA of the
    // tile's queries against the batch's representatives (same centring and
    // bounds as the member pairs) gives every query an interval
    // [dl, du] for d(q, Rc).  Then, per query:
    //   - theta_q <= du + (k-th member distance of c) for any cluster with
    //     at least k members (those k members are within that distance);
    //   - cluster c is needed only if dl - cmax(c) <= theta_q, and then only
    //     its members with d(s,Rc) in [dl - theta_q, du + theta_q]
    //     (triangle inequality), one contiguous run of the sorted members.
    // The tile streams, per cluster, the union of its queries' runs.
    // compacts every buffer of the tile holding more than `above` pairs (and
    // at least k); the rows are shared out over the four warps through shared
    // memory.  Called by the whole CTA.
    int *s_req = reinterpret_cast<int *>(s_n);
    int *s_kept = reinterpret_cast<int *>(s_e);
    float *s_uk = s_t;
    auto compact_rows = [&](int above) {
      const bool mine = valid && !ovf && n > above && n >= k;
      if (row_thread) s_req[tid] = mine ? n : 0;
      if (!__syncthreads_or(mine)) return;
      for (int rr = warp; warp < 4 && rr < cnt; rr += 4) {
        const int nn = s_req[rr];
        if (nn == 0) continue;
        const size_t ro = (row0 + rr) * cap;
        float uk;
        copy_entries(w_lu, w_pos, a.buf_lu + ro, a.buf_pos + ro, nn, lane);
        const int kept = compact_bounds(w_lu, w_pos, nn, k, whist, lane, &uk);
        copy_entries(a.buf_lu + ro, a.buf_pos + ro, w_lu, w_pos, kept, lane);
        if (lane == 0) {
          s_kept[rr] = kept;
          s_uk[rr] = uk;
        }
      }
      __syncthreads();
      if (mine) {
        const int kept = s_kept[tid];
        const float uk = s_uk[tid];
        n = kept;
        tau = fminf(tau, uk);
        th_q = fminf(th_q, sqrtf(uk) * (1.0f + tol));
        lim = min(cap - kTN, kept * KNN_TILE_GROW / 2 + 32);
        if (kept > cap - kTN) ovf = true;
      }
    };
    // the first batch holds the nearest clusters only: they tighten the
    // bounds before the rest of the list is decided
    const int nfirst = min(KNN_TILE_FIRST, nl);
    for (int jb = 0, nb = 0; jb < nl && ok; jb += nb) {
#if KNN_CHUNK_EXIT
      // the rest of the list is prunable for every query of the tile: its
      // nearest cluster's d(Rq, Rs) (the chunk of jb starts at or before
      // it), less the row's d(q, Rq) and the largest radius from there on,
      // beyond the row's bound (the filter's test, twice its margin)
      if (a.clb && jb > 0) {
        bool done = true;
        if (valid) {
          const float2 cb = a.clb[(size_t)qc * a.clb_stride + (jb >> 5)];
          done = cb.x - dq_row - cb.y > th_q + 2.0f * tol * (cb.x + dq_row + cb.y + th_q);
        }
        if (__syncthreads_and(done)) break;
      }
#endif
      nb = jb == 0 ? nfirst : min(kTN, nl - jb);
      stage_tile<NT>(
          sb, sc, KD, d, dp4,
          [&](int r) -> const float4 * {
            return r < nb ? a.sreps + (size_t)rl[jb + r] * dp4 : nullptr;
          },
          s_n, s_e, s_t);
      if (tid < nb) {
        const int c = rl[jb + tid];
        const int c0 = a.soff[c], sz = a.soff[c + 1] - c0;
        s_cmin[tid] = a.cmin[c];
        s_cmax[tid] = a.cmax[c];
        s_ck[tid] = sz >= k ? a.sdist[c0 + k - 1] : __int_as_float(0x7f800000);
        s_blo[tid] = 0x7f800000u;
        s_bhi[tid] = 0u;
      }
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (tid == 0) {
        for (int st = 0; st < KD / 16; st++) {
          const uint64_t ad = tc::make_desc(a_base + 256u * st, 128u, sbo);
          const uint64_t bd = tc::make_desc(b_base + 256u * st, 128u, sbo);
          tc::mma_bf16(tmem, ad, bd, idesc, st > 0);
        }
        tc::mma_commit(mbar);
      }
      if (row_thread)
        s_col[tid] = tid < nb ? make_float4(s_n[tid], sqrtf(s_e[tid]), sqrtf(s_t[tid]), 0.0f)
                              : make_float4(__int_as_float(0x7f800000), 0.0f, 0.0f, 0.0f);
      ok = tc::mbar_wait(mbar, phase);
      phase ^= 1u;
      ok = __syncthreads_and(ok) != 0;
      if (!ok) break;
      tc::fence_after_sync();
      const bool act = valid && !ovf;
      // pass 1: tighter theta_q from clusters with >= k members
      for (int cc = 0; warp < 4 && cc < nb; cc += 32) {  // TMEM lanes: warps 0-3
        float acc[32];
        tc::tmem_ld_32x32(lane_base + (uint32_t)cc, acc);
        if (act) {
#pragma unroll
          for (int jj = 0; jj < 32; jj++) {
            const float4 cv = s_col[cc + jj];
            const float base = na + cv.x;
            const float t2 = -2.0f * acc[jj];
            const float dl = __fmaf_rn(qa, cv.y, qb * cv.z);
            const float U = __fmaf_rn(base, 1.0f + kap, t2) + dl;
            const float ub = (sqrtf(fmaxf(U, 0.0f)) + s_ck[cc + jj]) * (1.0f + tol);
            if (cc + jj < nb) th_q = fminf(th_q, ub);
          }
        }
      }
      if (act) tau = fminf(tau, th_q * th_q * (1.0f + 4.0f * tol));
      // pass 2: the clusters each query needs and the union of their runs
      for (int cc = 0; warp < 4 && cc < nb; cc += 32) {  // TMEM lanes: warps 0-3
        float acc[32];
        tc::tmem_ld_32x32(lane_base + (uint32_t)cc, acc);
        if (act) {
#pragma unroll
          for (int jj = 0; jj < 32; jj++) {
            const int col = cc + jj;
            const float4 cv = s_col[col];
            const float base = na + cv.x;
            const float t2 = -2.0f * acc[jj];
            const float dl = __fmaf_rn(qa, cv.y, qb * cv.z);
            const float L = __fmaf_rn(base, 1.0f - kap, t2) - dl;
            const float U = __fmaf_rn(base, 1.0f + kap, t2) + dl;
            const float Dl = sqrtf(fmaxf(L, 0.0f)), Du = sqrtf(fmaxf(U, 0.0f));
            const float sl = tol * (Du + th_q + s_cmax[col]) + 1.17549435e-38f;
            if (col < nb && Dl - s_cmax[col] - sl <= th_q && Du + th_q + sl >= s_cmin[col]) {
              atomicMin(&s_blo[col], __float_as_uint(fmaxf(Dl - th_q - sl, 0.0f)));
              atomicMax(&s_bhi[col], __float_as_uint(Du + th_q + sl));
            }
          }
        }
      }
      tc::fence_before_sync();
      __syncthreads();  // TMEM and the member tile are reused below
      tc::fence_after_sync();
      // runs: the members of cluster tid whose d(s,Rc) is in [blo, bhi]
      {
        int lo = 0, len = 0;
        if (tid < nb && s_blo[tid] <= s_bhi[tid]) {
          const int c = rl[jb + tid];
          const float lo_v = __uint_as_float(s_blo[tid]), hi_v = __uint_as_float(s_bhi[tid]);
          int l = a.soff[c], h = a.soff[c + 1];
          while (l < h) {  // first member with d(s,Rc) >= lo_v
            const int md = (l + h) >> 1;
            if (a.sdist[md] < lo_v) l = md + 1;
            else h = md;
          }
          lo = l;
          h = a.soff[c + 1];
          while (l < h) {  // first member with d(s,Rc) > hi_v
            const int md = (l + h) >> 1;
            if (a.sdist[md] <= hi_v) l = md + 1;
            else h = md;
          }
          len = l - lo;
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += t;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        int before = 0;
        for (int w = 0; w < warp; w++) before += s_wsum[w];
        if (row_thread) {
          s_rlo[tid] = lo;
          s_roff[tid] = before + incl - len;
        }
        if (tid == kTM - 1) s_wmax[1] = (uint32_t)(before + incl);
      }
      __syncthreads();
      const int total = (int)s_wmax[1];
#if KNN_TILE_PROFILE
      if (tid == 0) {
        atomicAdd(&tile_prof[8], 1ull);
        atomicAdd(&tile_prof[10], (unsigned long long)total);
        if (jb == 0) {
          atomicAdd(&tile_prof[11], 1ull);
          atomicAdd(&tile_prof[12], (unsigned long long)nl);
        }
      }
#endif
      // the runs, concatenated, in chunks of kTN rows
      for (int o = 0; o < total; o += kTN) {
        const int nr = min(kTN, total - o);
        const bool last_of_first = jb == 0 && o + kTN >= total;
        stage_tile<NT>(
            sb, sc, KD, d, dp4,
            [&](int r) -> const float4 * {
              if (r >= nr) return nullptr;
              const int g = o + r;
              int l = 0, h = kTN - 1;  // last run starting at or before g
              while (l < h) {
                const int md = (l + h + 1) >> 1;
                if (s_roff[md] <= g) l = md;
                else h = md - 1;
              }
              const int p = s_rlo[l] + (g - s_roff[l]);
              s_pos[r] = p;
              return a.srows + (size_t)p * dp4;
            },
            s_n, s_e, s_t);
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        TILE_PROF(1);
        if (tid == 0) {
          for (int st = 0; st < KD / 16; st++) {
            const uint64_t ad = tc::make_desc(a_base + 256u * st, 128u, sbo);
            const uint64_t bd = tc::make_desc(b_base + 256u * st, 128u, sbo);
            tc::mma_bf16(tmem, ad, bd, idesc, st > 0);
          }
          tc::mma_commit(mbar);
        }
        // column scalars: |b|^2 (+inf on padding), |b - b~|, |b~|, position
        if (row_thread)
          s_col[tid] = tid < nr ? make_float4(s_n[tid], sqrtf(s_e[tid]), sqrtf(s_t[tid]),
                                              __int_as_float(s_pos[tid]))
                                : make_float4(__int_as_float(0x7f800000), 0.0f, 0.0f, 0.0f);
        ok = tc::mbar_wait(mbar, phase);
        phase ^= 1u;
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
        tc::fence_after_sync();
        TILE_PROF(2);
        for (int cc = 0; warp < 4 && cc < nr; cc += 32) {  // TMEM lanes: warps 0-3
          float acc[32];
          tc::tmem_ld_32x32(lane_base + (uint32_t)cc, acc);
          if (valid && !ovf) {
#pragma unroll
            for (int jj = 0; jj < 32; jj++) {
              const float4 cv = s_col[cc + jj];
              const float base = na + cv.x;
              const float t2 = -2.0f * acc[jj];
              const float dl = __fmaf_rn(qa, cv.y, qb * cv.z);
              const float L = __fmaf_rn(base, 1.0f - kap, t2) - dl;
              if (L <= tau && n < cap) {
                const float U = __fmaf_rn(base, 1.0f + kap, t2) + dl;
                my_lu[n] = make_float2(fmaxf(L, 0.0f), fmaxf(U, 0.0f));
                my_pos[n] = __float_as_int(cv.w);
                n++;
              }
            }
          }
        }
        if (valid) pairs += (unsigned long long)nr;
        TILE_PROF(3);
        // buffers past their limit are compacted (tightening tau); after the
        // first batch every buffer holding k pairs is, so that the next
        // batch's runs use the tightened bounds
        compact_rows(last_of_first ? k - 1 : lim);
        TILE_PROF(4);
        tc::fence_before_sync();
        __syncthreads();  // the member tile, TMEM and column scalars are reused
        tc::fence_after_sync();
        TILE_PROF(5);
      }
    }
    if (!ok) break;
    TILE_PROF(5);

#if KNN_TILE_PROFILE
    if (valid) {
      atomicAdd(&tile_prof[13], (unsigned long long)(sqrtf(tau) * 1000.0f));
      atomicAdd(&tile_prof[15], 1ull);
    }
#endif
    // finish the tile's queries, shared out over the warps (all of them when
    // their state fits the free tile region): exact re-ranking and the FP64
    // boundary, on a shared-memory copy of each query's buffer
    if (row_thread) {
      s_req[tid] = n;
      s_kept[tid] = ovf ? 1 : 0;
    }
    __syncthreads();
    for (int row = warp; warp < nrw && row < cnt; row += nrw) {
      const int nn = s_req[row];
      bool fb = s_kept[row] != 0;
      const int slot = s0 + row;
      const int64_t q = a.qorder[slot];
      const size_t ro = (row0 + row) * cap;
      int m1 = nn;
      if (!fb) {
        copy_entries(w_lu, w_pos, a.buf_lu + ro, a.buf_pos + ro, m1, lane);
        if (m1 > k) {
          float uk;
          m1 = compact_bounds(w_lu, w_pos, m1, k, whist, lane, &uk);
        }
      }
      // exact FP32 keys, written over the bound pairs
      uint64_t *keys = reinterpret_cast<uint64_t *>(w_lu);
      const float *qf = reinterpret_cast<const float *>(a.qrows + (size_t)q * dp4);
      for (int c = lane; c < dp4; c += 32) wq[c] = a.qrows[(size_t)q * dp4 + c];
      __syncwarp();
      if (!fb) {
        for (int e = lane; e < m1; e += 32) {
          const int p = w_pos[e];
          const float d2 = dist2_cols(wq, a.srows + (size_t)p * dp4, d);
          keys[e] = make_key(d2, a.sidx[p]);
        }
        if (lane == 0) refined += (unsigned long long)m1;
        __syncwarp();
      }
      // the k smallest keys plus every key inside the FP32 band of the k-th,
      // sorted: keys[0..m2).  Up to 128 keys are sorted directly in registers;
      // larger sets are first cut down by a selection of the k-th key.
      int m2 = m1;
      bool sorted = false;
      if (!fb && m1 <= 128) {
        if (m1 <= 32) sort_keys_in_registers<1>(keys, m1, lane);
        else if (m1 <= 64) sort_keys_in_registers<2>(keys, m1, lane);
        else sort_keys_in_registers<4>(keys, m1, lane);
        sorted = true;
        if (m1 > k) {
          const float Dk = key_d2(keys[k - 1]);
          const float lim2 = band_hi(Dk, d);
          int w = 0;
          for (int b0 = 0; b0 < m1; b0 += 32) {
            const int e = b0 + lane;
            w += __popc(__ballot_sync(kFull, e < m1 && key_d2(keys[e]) <= lim2));
          }
          m2 = w;
        }
      } else if (!fb && m1 > k) {
        // keys up to band_hi of (an upper bound of) the k-th; the band itself
        // is settled on the sorted keys below
#if KNN_LINEAR_SELECT
        const float Dk = __uint_as_float(warp_kth_upper_u32(
            reinterpret_cast<const uint32_t *>(keys) + 1, 2, m1, k, whist, lane));
#else
        const float Dk = key_d2(warp_select_kth(keys, m1, k, whist, lane));
#endif
        const float lim2 = band_hi(Dk, d);
        int w = 0;
        for (int b0 = 0; b0 < m1; b0 += 32) {
          const int e = b0 + lane;
          const uint64_t key = e < m1 ? keys[e] : kKeyMax;
          const bool keep = e < m1 && key_d2(key) <= lim2;
          const unsigned bm = __ballot_sync(kFull, keep);
          __syncwarp();
          if (keep) keys[w + __popc(bm & ((1u << lane) - 1u))] = key;
          w += __popc(bm);
        }
        __syncwarp();
        m2 = w;
      }
      int np2 = 32;
      while (np2 < (sorted ? m1 : m2)) np2 <<= 1;
      if (!fb && np2 > cap) fb = true;
      if (!fb) {
        if (!sorted) {
#if KNN_BIN_SORT
          // binned counting sort where its scratch fits behind the keys
          sorted = m2 <= 256 && np2 + m2 <= cap &&
                   warp_bin_sort<8>(keys, m2, keys + np2, whist, lane);
#endif
          if (!sorted) {
            for (int e = m2 + lane; e < np2; e += 32) keys[e] = kKeyMax;
            __syncwarp();
            smem_bitonic_sort_rt(keys, np2, lane);
          }
        }
        if (m2 > k) {
          // keys at or above Dk - band were ranked in FP32 only to within
          // rounding: order them again by (FP64 d^2, index)
          const float Dk = key_d2(keys[k - 1]);
          const float lo_v = band_lo(Dk, d);
          int lo = 0;
          for (int b0 = 0; b0 < m2; b0 += 32) {
            const int e = b0 + lane;
            lo += __popc(__ballot_sync(kFull, e < m2 && key_d2(keys[e]) < lo_v));
          }
          const int bsz = m2 - lo;
          if (2 * bsz > cap || np2 + bsz > cap) {
            fb = true;
          } else {
            double *d64 = reinterpret_cast<double *>(w_pos);
            uint64_t *perm = keys + np2;
            for (int e = lane; e < bsz; e += 32) {
              const int32_t id = key_idx(keys[lo + e]);
              d64[e] = dist2_f64(
                  qf, reinterpret_cast<const float *>(a.rrows + (size_t)id * dp4), d);
            }
            __syncwarp();
            for (int e = lane; e < bsz; e += 32) {
              const double de = d64[e];
              const int32_t ie = key_idx(keys[lo + e]);
              int rank = 0;
              for (int f = 0; f < bsz; f++) {
                const double df = d64[f];
                const int32_t iff = key_idx(keys[lo + f]);
                rank += (df < de || (df == de && iff < ie)) ? 1 : 0;
              }
              perm[rank] = keys[lo + e];
            }
            __syncwarp();
            for (int e = lane; e < bsz; e += 32) keys[lo + e] = perm[e];
            __syncwarp();
            if (lane == 0) rechecks += (unsigned long long)bsz;
          }
        }
      }
      if (fb) {
        if (lane == 0) {
          a.fb_slots[atomicAdd(a.fb_count, 1u)] = slot;
          fallbacks++;
        }
      } else {
        int32_t *oi = a.out_idx + (size_t)q * k;
        float *od = a.out_dist + (size_t)q * k;
        for (int t = lane; t < k; t += 32) {
          const uint64_t key = t < m2 ? keys[t] : kKeyMax;
          const bool none = key == kKeyMax;
          oi[t] = none ? -1 : key_idx(key);
          const float d2 = key_d2(key);
          od[t] = none ? __int_as_float(0x7f800000) : (a.squared ? d2 : sqrtf(d2));
        }
      }
      __syncwarp();
    }
    TILE_PROF(6);
    __syncthreads();  // the next tile overwrites the query tile and centre
    TILE_PROF(7);
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
#if KNN_TILE_PROFILE
  if (tid == 0)
    for (int i = 0; i < 8; i++) atomicAdd(&tile_prof[i], prof[i]);
#endif
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(kFull, pairs, o);
  if (lane == 0) {
    atomicAdd(&a.counters[0], pairs);
    atomicAdd(&a.counters[1], refined);
    atomicAdd(&a.counters[2], rechecks);
    atomicAdd(&a.counters[3], fallbacks);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTN);
}

int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

bool tile_search_supported(int d, int k, int margin) {
  return d >= 16 && d <= 256 && k >= 1 && k <= KNN_MAX_K && margin >= 0 && margin <= 4096;
}

// Shared memory of one CTA for a per-query buffer of `cap` entries.
static size_t tile_smem_bytes(int KD, int cap) {
  return tiles_bytes(KD) + (size_t)KD * 4 + (size_t)kTN * 16 + 11 * (size_t)kTN * 4 +
         (size_t)(2 * kTM / 32 + 4) * 4 + 4 * 256 * 4 + 8 + 4 + 16 + 16 + 4 * (size_t)cap * 12 +
         4 * (size_t)(KD / 4) * 16;
}

// Threads per CTA: 2 kTM where the re-ranking state of four more warps fits
// the tile region (dp4 <= KD / 4), kTM otherwise.
static int tile_threads(int KD, int cap) {
  const size_t wstate = (size_t)cap * 12 + (size_t)(KD / 4) * 16 + 256 * 4;
  return 4 * wstate <= tiles_bytes(KD) ? 2 * kTM : kTM;
}

template <int NT>
static int set_tile_attributes(size_t smem) {
  KNN_CUDA_TRY(cudaFuncSetAttribute(tile_search_kernel<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the whole unified L1 as shared memory: the CTAs per SM are then set by
  // shared memory alone (the default split allowed one)
  KNN_CUDA_TRY(cudaFuncSetAttribute(tile_search_kernel<NT>,
                                    cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
  return KNN_OK;
}

int tile_search_geometry(int d, int k, int margin, int num_sms, int *grid, int *cap, int *P,
                         size_t *smem) {
  const int KD = std::max(16, pow2_at_least(d));
  *P = std::max(32, pow2_at_least(k + 64));
  // each query keeps up to cap bound pairs; smaller if shared memory is short
  *cap = 4 * (k + margin) + kTN;
  if (tile_smem_bytes(KD, *cap) > 227 * 1024) *cap = 2 * (k + margin) + kTN;
  *cap = std::max(*cap, *P);
  // at least 48 KB: no more than four CTAs (4 x 128 TMEM columns) per SM
  *smem = std::max<size_t>(tile_smem_bytes(KD, *cap), 48 * 1024 + 1024);
  if (*smem > 227 * 1024) return KNN_EINVAL;
  const int nt = tile_threads(KD, *cap);
  const int rc = nt == kTM ? set_tile_attributes<kTM>(*smem) : set_tile_attributes<2 * kTM>(*smem);
  if (rc != KNN_OK) return rc;
  // CTAs per SM by shared memory (1 KB of it reserved per CTA); the
  // persistent CTAs that find no SM slot simply start later
  int dev = 0, smem_sm = 0;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  KNN_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  int per_sm = (int)((size_t)smem_sm / (*smem + 1024));
  // and by registers: 128 per thread, so four CTAs of kTM threads, two of 2 kTM
  per_sm = std::max(1, std::min(per_sm, nt == kTM ? 4 : 2));
  *grid = num_sms * per_sm;
  return KNN_OK;
}

int launch_tile_list(const int32_t *qoff, int Rq, int c_base, int32_t *tiles, int32_t *ntiles,
                     cudaStream_t s) {
  tile_list_kernel<<<1, 1024, 0, s>>>(qoff, Rq, c_base, tiles, ntiles);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_tile_search(const TileArgs &a, int grid, size_t smem, cudaStream_t s) {
  if (tile_threads(a.KD, a.cap) == kTM)
    tile_search_kernel<kTM><<<grid, kTM, smem, s>>>(a);
  else
    tile_search_kernel<2 * kTM><<<grid, 2 * kTM, smem, s>>>(a);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

}  // namespace knnsweet

#if KNN_TILE_PROFILE
// Profiling hook: copies and clears the phase timers (8 counters) and the
// pruning counters (8 more).
extern "C" int knnsweet_tile_profile(unsigned long long *out) {
  if (cudaMemcpyFromSymbol(out, knnsweet::tile_prof, 16 * sizeof(unsigned long long)) !=
      cudaSuccess)
    return -3;
  unsigned long long z[16] = {};
  return cudaMemcpyToSymbol(knnsweet::tile_prof, z, sizeof z) == cudaSuccess ? 0 : -3;
}
#endif
