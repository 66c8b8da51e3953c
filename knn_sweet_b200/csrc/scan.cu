// scan.cu -- the per-query pruned scan (replaces KNNQuery_base,
// src/knnjoin.cu:762-858, and the small-M KNNQuery + final merge,
// src/knnjoin.cu:859-979).
//
// One warp per query, persistent blocks pulling query slots from an atomic
// counter in query-cluster order (the reference's reorder_members,
// knnjoin.cu:114-124, 768), so neighbouring warps walk the same candidate
// list.  For the surviving reference clusters Rs of the query's cluster,
// 32 at a time:
//   - each lane computes D = d(q, Rs) and drops its cluster if
//     D - radius(Rs) > theta or D + theta < smallest member distance: no
//     member can be within theta (the reference's first-member `break`,
//     knnjoin.cu:797); the survivors are visited nearest first (a warp sort
//     on D), so the running k-th distance theta falls early.
//   - Members are stored contiguously, ascending by d(s, Rs).  Members within
//     theta of q satisfy |D - d(s,Rs)| <= theta (knnjoin.cu:796-801), a
//     contiguous band.  A warp-wide 32-ary search finds (to within 31
//     members) where the band starts; the warp walks it 32 members per step
//     with coalesced row loads and stops at the first step past its upper
//     end (re-evaluated with the current theta).
//   - Exact FP32 distances go through the warp top-k: k <= 24 a sorted
//     register list (one key per lane) merged by shuffle networks; larger k
//     an unsorted candidate set in shared memory, compacted to the keys up to
//     the FP32 band of (an upper bound of) the k-th distance when it fills,
//     sorted once at the end of the query.  This replaces the per-thread
//     insertion into an 8 KB local-memory array (knnjoin.cu:774, 813-845).
//   - The k-th boundary is then settled in FP64 (see TopKBase).
// Bounds are widened by a rounding slack (bound_tol) so that FP32 rounding
// never prunes a point that the FP32 distances would rank in the top k.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "warp_select.cuh"

namespace knnsweet {

// Shared part of the top-k variants: the append buffer, the admission
// threshold and what the FP64 re-check of the k-th boundary needs.
//
// The neighbour set must be the one an FP64 join gives.  Keys are FP32
// (d^2, index) words, which rank two points differently from FP64 only when
// both lie inside the FP32 rounding band of the k-th squared distance
// (band_lo / band_hi).  So the admission threshold, once k keys are in, is
// band_hi of the current k-th value (every point that may still belong to
// the final band is admitted and never pruned), compactions keep every key up
// to that value, and `lostmin` records the smallest FP32 d^2 of any key that
// had to be dropped for lack of room while it could still lie in the final
// band.  At the end of the query the band is re-decided in FP64
// (band_resolve_fp64); a query that lost a band key goes to the band kernel
// instead.
//
// Register budget: the dimension comes from the kernel parameters where it is
// needed and `lostmin` lives in a shared-memory word of the warp, so neither
// occupies a register through the scan loop.
//
// The warp's shared-memory slot holds, at fixed key offsets behind the
// buffer, `lostmin` (the smallest FP32 d^2 dropped for lack of room, +inf:
// none), the current query's statistics words (kStat*, updated by lane 0)
// and the query's slot, row and cluster (kSide*, needed only when the query
// starts and ends): kept out of registers, which the scan loop needs.
enum {
  kStatPushed = 0, kStatMerges, kStatVisited, kStatPruned, kStatChecked,
  kSideSlot, kSideQuery, kSideCluster, kSideDq, kStatWords
};
constexpr int kStatKeys = (kStatWords + 1) / 2;  // 64-bit words they take

template <int kLostOff, int kStatOff>
struct TopKBase {
  uint64_t *buf;  // append buffer (shared memory)
  int nbuf, nlist, k;
  // a candidate (d^2, index) enters iff d^2 <= thr_d2: the threshold key
  // (thr_d2, 0xffffffff) lies above every key with that distance word
  float thr_d2;
  float theta;    // distance matching thr (bound for the pruning tests)

  __device__ __forceinline__ float *lostmin() const {
    return reinterpret_cast<float *>(buf + kLostOff);
  }
  __device__ __forceinline__ unsigned *stat() const {
    return reinterpret_cast<unsigned *>(buf + kStatOff);
  }
  __device__ __forceinline__ void count(int which, unsigned v, int lane) const {
    if (lane == 0) stat()[which] += v;
  }

  __device__ __forceinline__ void reset_threshold(float th0, int lane) {
    nbuf = 0;
    nlist = 0;
    theta = th0;
    if (lane == 0) *lostmin() = __int_as_float(0x7f800000);
    // admits every d^2 <= th0^2, whatever the index
    thr_d2 = th0 * th0;
  }
  // threshold once the k-th squared distance is T: the FP32 band above it
  __device__ __forceinline__ void set_band_threshold(float T, int d) {
    const float W = band_hi(T, d);
    thr_d2 = W;
    theta = sqrtf(W);
  }
  // a dropped key's distance word (NaN from an empty key is ignored)
  __device__ __forceinline__ void note_lost(uint32_t d2bits, int lane) {
    const float v = __uint_as_float(__reduce_min_sync(kFull, d2bits));
    __syncwarp();
    if (lane == 0) *lostmin() = fminf(*lostmin(), v);
    __syncwarp();
  }
};

// Small k: the sorted list of the best keys lives in registers
// (one key per lane), with the FP32 band of the k-th kept behind it as far as
// the 32 slots allow.
template <int E>
struct RegTopK : TopKBase<64 * E + 2, 64 * E + 3> {
  using B = TopKBase<64 * E + 2, 64 * E + 3>;
  using B::buf, B::nbuf, B::nlist, B::k, B::count, B::note_lost, B::set_band_threshold,
      B::reset_threshold;
  static constexpr int L = 32 * E;
  static constexpr int kCap = L;  // candidate buffer capacity
  // append buffer (L keys), L doubles for the FP64 band, 2 pivot words,
  // lostmin, statistics
  static constexpr int kSmemKeys = 2 * L + 3 + kStatKeys;
  static constexpr int kBandScratch = L, kPivot = 2 * L;
  uint64_t v[E];

  __device__ __forceinline__ int cap() const { return kCap; }

  __device__ __forceinline__ void init(uint64_t *wsm) { buf = wsm; }

  __device__ __forceinline__ void reset(float th0, int lane) {
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = kKeyMax;
    reset_threshold(th0, lane);
  }

  __device__ __forceinline__ void make_room(int lane, int d) { flush(lane, d); }
  // end of the query: pending candidates merged into the list
  __device__ __forceinline__ void finish(int lane, int d) { flush(lane, d); }

  __device__ __forceinline__ void flush(int lane, int d) {
    if (nbuf == 0) return;
    __syncwarp();
    uint64_t b[E];
#pragma unroll
    for (int j = 0; j < E; j++) {
      const int p = j * 32 + lane;  // any order: the buffer gets sorted
      b[j] = p < nbuf ? buf[p] : kKeyMax;
    }
    __syncwarp();
    reg_bitonic_sort<E>(b, lane);
    // v ascending, b ascending: min(v[i], b[L-1-i]) holds the L smallest of
    // both as a bitonic sequence; the larger of each pair is dropped
    uint32_t lost = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < E; j++) {
      const uint64_t o = shfl64(b[E - 1 - j], 31 - lane);
      lost = min(lost, (uint32_t)(umax64(v[j], o) >> 32));
      v[j] = umin64(v[j], o);
    }
    note_lost(lost, lane);
    reg_bitonic_merge<E>(v, lane);
    nlist = min(k, nlist + nbuf);
    count(kStatMerges, 1, lane);
    nbuf = 0;
    if (nlist == k) {
      const int kl = (k - 1) / E, kj = (k - 1) % E;
      uint64_t mine = kKeyMax;
#pragma unroll
      for (int j = 0; j < E; j++)
        if (j == kj) mine = v[j];
      const float T = key_d2(shfl64(mine, kl));
      // keys behind the k-th stay only inside its band (the ones dropped
      // here are above band_hi of a k-th that can only fall)
      const float hi = band_hi(T, d);
#pragma unroll
      for (int j = 0; j < E; j++)
        if (E * lane + j >= k && key_d2(v[j]) > hi) v[j] = kKeyMax;
      set_band_threshold(T, d);
    }
  }

  // The candidates, sorted, into buf[0..n); returns n.
  __device__ __forceinline__ int sorted(int lane, int) {
    __syncwarp();
    int n = 0;
#pragma unroll
    for (int j = 0; j < E; j++) {
      buf[E * lane + j] = v[j];
      n += __popc(__ballot_sync(kFull, v[j] != kKeyMax));
    }
    __syncwarp();
    return n;
  }
};

// Bitonic sort of L keys in shared memory, ascending, by one warp.
template <int L>
__device__ __forceinline__ void smem_bitonic_sort(uint64_t *s, int lane) {
#pragma unroll 1
  for (int size = 2; size <= L; size <<= 1) {
#pragma unroll 1
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
      for (int t0 = 0; t0 < (L / 2 + 31) / 32; t0++) {
        const int t = t0 * 32 + lane;
        if (t < L / 2) {
          const int i = 2 * t - (t & (stride - 1));
          const int j = i + stride;
          const bool up = (i & size) == 0;
          const uint64_t a = s[i], b = s[j];
          if ((a > b) == up) {
            s[i] = b;
            s[j] = a;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Top-k as an unsorted candidate set in shared memory (capacity 2L).  When it
// fills, the k-th smallest squared distance T is found by a radix selection
// and the set keeps every key up to band_hi(T); the k results are sorted
// once, at the end of the query.
#ifndef KNN_TOPK_EARLY
#define KNN_TOPK_EARLY 160
#endif

template <int LL>
struct SelectTopK : TopKBase<2 * LL + 128, 2 * LL + 129> {
  using B = TopKBase<2 * LL + 128, 2 * LL + 129>;
  using B::buf, B::nbuf, B::nlist, B::k, B::count, B::note_lost, B::set_band_threshold,
      B::reset_threshold;
  static constexpr int L = LL;          // final sort length (pow2 >= k)
  static constexpr int kCap = 2 * LL;   // candidate capacity
  // keys, 256-word histogram, lostmin, statistics
  static constexpr int kSmemKeys = 2 * LL + 129 + kStatKeys;
  // after the final sort: LL doubles for the FP64 band behind the sorted
  // keys, the pivot in the histogram's words
  static constexpr int kBandScratch = LL, kPivot = 2 * LL;
  __device__ __forceinline__ uint32_t *hist() const {
    return reinterpret_cast<uint32_t *>(buf + 2 * LL);
  }

  // A compaction once k + kEarly candidates are in (capacity permitting)
  // tightens the threshold sooner.  k = 200 self-join scan: capacity only
  // 5.06 ms; kEarly 64: 5.12, 96: 4.94, 128: 4.89, 160: 4.90, 256: 4.97
  // (with the compaction before the end-of-query selection: 96: 4.86,
  // 128 to 192: 4.76-4.78).
  static constexpr int kEarly = KNN_TOPK_EARLY;
  __device__ __forceinline__ int cap() const { return k + kEarly < kCap ? k + kEarly : kCap; }

  __device__ __forceinline__ void init(uint64_t *wsm) { buf = wsm; }

  __device__ __forceinline__ void reset(float th0, int lane) { reset_threshold(th0, lane); }

  // Reduce the set to its k smallest keys (no-op with k or fewer) when ties
  // leave no room otherwise; the keys it drops go into lostmin.
  __device__ __forceinline__ void flush(int lane, int d) {
    if (nbuf <= k) return;
    __syncwarp();
    const uint64_t kth = warp_select_kth(buf, nbuf, k, hist(), lane);
    __syncwarp();
    int w = 0;
    uint32_t lost = 0xffffffffu;
    for (int b0 = 0; b0 < nbuf; b0 += 32) {
      const int i = b0 + lane;
      const uint64_t v = i < nbuf ? buf[i] : kKeyMax;
      const bool keep = i < nbuf && v <= kth;
      if (i < nbuf && !keep) lost = min(lost, (uint32_t)(v >> 32));
      const unsigned bm = __ballot_sync(kFull, keep);
      __syncwarp();
      if (keep) buf[w + __popc(bm & ((1u << lane) - 1))] = v;
      w += __popc(bm);
    }
    __syncwarp();
    note_lost(lost, lane);
    nbuf = w;  // == k
    nlist = k;
    count(kStatMerges, 1, lane);
    set_band_threshold(key_d2(kth), d);
  }

  // Room for more candidates while the query runs: keep every key whose
  // squared distance is at most band_hi of the k-th smallest one T -- at
  // least k keys, ties and the FP32 band included -- found by a 32-bit
  // selection on the keys' distance words (on data with many equal distances
  // a 64-bit selection spends most of its passes on the index bits of the
  // ties).  Falls back to the exact k-key flush when ties fill the buffer.
  __device__ __forceinline__ void make_room(int lane, int d) {
    if (nbuf <= k) return;
    __syncwarp();
#if KNN_LINEAR_SELECT
    // an upper bound of the k-th: the threshold it gives admits a little more
    const uint32_t T = warp_kth_upper_u32(reinterpret_cast<const uint32_t *>(buf) + 1, 2,
                                          nbuf, k, hist(), lane);
#else
    const uint32_t T = warp_select_kth_u32(reinterpret_cast<const uint32_t *>(buf) + 1, 2,
                                           nbuf, k, hist(), lane);
#endif
    const uint32_t W = __float_as_uint(band_hi(__uint_as_float(T), d));
    int w = 0;
    for (int b0 = 0; b0 < nbuf; b0 += 32) {
      const int i = b0 + lane;
      const uint64_t v = i < nbuf ? buf[i] : kKeyMax;
      const bool keep = i < nbuf && (uint32_t)(v >> 32) <= W;
      const unsigned bm = __ballot_sync(kFull, keep);
      __syncwarp();
      if (keep) buf[w + __popc(bm & ((1u << lane) - 1))] = v;
      w += __popc(bm);
    }
    __syncwarp();
    nbuf = w;
    if (w > kCap - 32) {
      flush(lane, d);
      return;
    }
    count(kStatMerges, 1, lane);
    nlist = k;
    set_band_threshold(__uint_as_float(T), d);
  }

  // End of the query: nothing to do before sorted().
  __device__ __forceinline__ void finish(int, int) {}

  // The candidates, sorted, into buf[0..n); returns n.  Up to L keys are
  // sorted as they are; beyond that a band-inclusive compaction first, and
  // the exact k-key flush only if ties still leave more than L.
  __device__ __forceinline__ int sorted(int lane, int d) {
    if (nbuf > LL) make_room(lane, d);
    if (nbuf > LL) flush(lane, d);
    __syncwarp();
    if constexpr (LL <= 128) {
      // sorted in registers (E keys per lane; shuffles for the cross-lane
      // strides): lane l ends up with positions E*l .. E*l+E-1.  (At L = 256
      // the eight keys per lane spilled under the kernel's register cap and
      // measured slower than the shared-memory sort.)
      constexpr int E = LL / 32;
      uint64_t x[E];
#pragma unroll
      for (int j = 0; j < E; j++) {
        const int p = j * 32 + lane;  // any order: the keys get sorted
        x[j] = p < nbuf ? buf[p] : kKeyMax;
      }
      __syncwarp();
      reg_bitonic_sort<E>(x, lane);
#pragma unroll
      for (int j = 0; j < E; j++) buf[E * lane + j] = x[j];
    } else {
      // binned counting sort (k = 200 self-join scan: 4.45 ms with the
      // bitonic network alone); the network where equal distances crowd a bin
#if KNN_BIN_SORT
      if constexpr (LL <= 256)  // the bin tags of 8 keys per lane stay in registers
        if (warp_bin_sort<LL / 32>(buf, nbuf, buf + LL, hist(), lane)) return nbuf;
#endif
      for (int i = nbuf + lane; i < LL; i += 32) buf[i] = kKeyMax;
      __syncwarp();
      smem_bitonic_sort<LL>(buf, lane);
    }
    __syncwarp();
    return nbuf;
  }
};

// Offer one candidate per lane, warp-collective: the lanes with `pass` set
// (squared distance v at most the threshold's distance word, so that the key
// (v, idx) lies below the threshold key) append their keys.
template <class TK>
__device__ __forceinline__ void topk_offer(TK &tk, bool pass, float v, int32_t idx, int lane,
                                           int d) {
  unsigned b = __ballot_sync(kFull, pass);
  if (b == 0) return;
  int cnt = __popc(b);
  if (tk.nbuf + cnt > tk.cap()) {
    tk.make_room(lane, d);
    pass = pass && v <= tk.thr_d2;
    b = __ballot_sync(kFull, pass);
    cnt = __popc(b);
  }
  if (pass) tk.buf[tk.nbuf + __popc(b & ((1u << lane) - 1))] = make_key(v, idx);
  tk.nbuf += cnt;
  tk.count(kStatPushed, cnt, lane);
}

// Whether every FP32 squared distance of the join is exact (both sides hold
// small integers), so that FP32 keys rank exactly like FP64 ones.
__device__ __forceinline__ bool fp32_exact(const ScanArgs &a) {
  return a.inexact_r && a.inexact_q && (*a.inexact_r | *a.inexact_q) == 0;
}

// A query's starting k-th distance bound.  theta0 of its cluster is the k-th
// smallest of rq + d(Rq,Rs) + d(s,Rs) over the reference points s, rq the
// cluster's radius; the same k points lie within dq + d(Rq,Rs) + d(s,Rs) of a
// query at distance dq <= rq from the representative, so theta0 - (rq - dq),
// widened by the rounding slack, bounds that query's k-th distance too and
// starts its scan tighter.
#ifndef KNN_QUERY_THETA0
#define KNN_QUERY_THETA0 1
#endif
__device__ __forceinline__ float query_theta0(const ScanArgs &a, int64_t slot, int qc, float tol) {
  float th = a.theta0[qc];
  if (KNN_QUERY_THETA0 && a.qrad && a.qkeys) {
    const float rq = a.qrad[qc], dq = __uint_as_float((uint32_t)a.qkeys[slot]);
    const float cut = (rq - dq) - tol * (rq + dq + th);
    if (cut > 0.0f) th -= cut;
  }
  return th;
}

// FP64 re-decision of one query's k-th boundary, by one warp.  s[0..n) holds
// the query's candidate keys sorted ascending, n > k; s[0..nlo) lie below the
// FP32 band of the k-th (band_lo(Dk) .. band_hi(Dk)), s[nlo..nhi) inside it,
// nhi > k, and every point inside the band is among them.  Keys below the
// band are in the FP64 top k, keys above it are not; the band's keys are
// ranked by (FP64 d^2, index) and the best k - nlo of them kept in place, in
// their FP32 order, so that s[0..k) is the FP64 join's neighbour set.  (The
// reference decides this boundary by a strict-less insertion of FP32
// distances, src/knnjoin.cu:815-820.)  qf: the query row; rrows: the
// reference rows in original order (keys carry original indices); dbl:
// scratch for nhi - nlo doubles; piv: 2 words.  Inlined: as an out-of-line
// call (for the few queries that need it) it cost the k = 200 self-join scan
// 8 % (5.15 against 4.82 ms), the call's register saves on every query.
__device__ __forceinline__ void band_resolve_fp64(uint64_t *s, int nlo, int nhi, int k, int d,
                                               int dp4, const float *__restrict__ qf,
                                               const float4 *__restrict__ rrows, double *dbl,
                                               uint64_t *piv, int lane) {
  const int nb = nhi - nlo, need = k - nlo;
  for (int e = lane; e < nb; e += 32) {
    const int32_t id = key_idx(s[nlo + e]);
    dbl[e] = dist2_f64(qf, reinterpret_cast<const float *>(rrows + (int64_t)id * dp4), d);
  }
  __syncwarp();
  // the need-th smallest (FP64 d^2, index) of the band (ranks are distinct)
  for (int e = lane; e < nb; e += 32) {
    const double de = dbl[e];
    const int32_t ie = key_idx(s[nlo + e]);
    int rank = 0;
    for (int f = 0; f < nb; f++) rank += f64_key_less(dbl[f], key_idx(s[nlo + f]), de, ie);
    if (rank == need - 1) {
      piv[0] = (uint64_t)__double_as_longlong(de);
      piv[1] = (uint64_t)(uint32_t)ie;
    }
  }
  __syncwarp();
  const double pd = __longlong_as_double((long long)piv[0]);
  const int32_t pi = (int32_t)piv[1];
  // keep the band's keys up to the pivot, in place, order preserved
  int w = nlo;
  for (int b0 = 0; b0 < nb; b0 += 32) {
    const int e = b0 + lane;
    const uint64_t key = e < nb ? s[nlo + e] : kKeyMax;
    const bool keep = e < nb && !f64_key_less(pd, pi, dbl[e], key_idx(key));
    const unsigned bm = __ballot_sync(kFull, keep);
    __syncwarp();
    if (keep) s[w + __popc(bm & ((1u << lane) - 1))] = key;
    w += __popc(bm);
  }
  __syncwarp();
}

// End of one query of the warp scan: sorts the candidates, settles the k-th
// boundary in FP64 unless the join's FP32 distances are exact (or, when a key of its band was dropped for lack of room,
// hands the query to the band kernel: the last output slot then carries the
// number of keys below the band and the FP32 k-th value), writes the k
// results.  Returns the FP64 distances evaluated.
template <class TK>
__device__ __forceinline__ unsigned emit_query(TK &tk, const ScanArgs &a, int32_t slot, int64_t q,
                                               int qc, int lane) {
  const int n = tk.sorted(lane, a.d);
  const bool exact32 = fp32_exact(a);
  uint64_t *s = tk.buf;
  const int k = a.k;
  bool defer = false;
  int nlo = 0;
  float Dk = 0.0f;
  unsigned checked = 0;
  if (n >= k && !exact32) {  // exact FP32 distances: the (d^2, index) order is FP64's
    Dk = key_d2(s[k - 1]);
    const float lo = band_lo(Dk, a.d), hi = band_hi(Dk, a.d);
    int nhi = 0;
    for (int b0 = 0; b0 < n; b0 += 32) {
      const int e = b0 + lane;
      const float v = e < n ? key_d2(s[e]) : __int_as_float(0x7f800000);
      nlo += __popc(__ballot_sync(kFull, v < lo));
      nhi += __popc(__ballot_sync(kFull, v <= hi));
    }
    if (*tk.lostmin() <= hi) {
      defer = true;
    } else if (nhi > k) {
      band_resolve_fp64(s, nlo, nhi, k, a.d, a.dp4,
                        reinterpret_cast<const float *>(a.qrows + q * a.dp4), a.rrows,
                        reinterpret_cast<double *>(s + TK::kBandScratch), s + TK::kPivot, lane);
      checked = (unsigned)(nhi - nlo);
    }
  }
  int32_t *oi = a.out_idx + q * k;
  float *od = a.out_dist + q * k;
  const int32_t base = a.qc_ref_base ? (int32_t)a.qc_ref_base[qc] : 0;
  for (int t = lane; t < k; t += 32) {
    const uint64_t key = t < n ? s[t] : kKeyMax;
    const bool none = key == kKeyMax;
    if (defer && t == k - 1) {
      oi[t] = nlo;
      od[t] = Dk;
    } else {
      oi[t] = none ? -1 : key_idx(key) - base;
      od[t] = none ? __int_as_float(0x7f800000) : (a.squared ? key_d2(key) : sqrtf(key_d2(key)));
    }
  }
  if (defer && lane == 0) a.unres_slot[atomicAdd(a.unres_count, 1u)] = slot;
  __syncwarp();
  return checked;
}

// ---------------------------------------------------------------------------
// Query rows.  IDXROW: the reference rows carry their original index in the
// last pad float (d < 4*DP4), which the distance then skips.
// ---------------------------------------------------------------------------
template <int DP4, bool IDXROW>
struct QueryRow {
  float4 v[DP4];
  __device__ __forceinline__ void load(const float4 *__restrict__ rows, int64_t q, int,
                                       float4 *) {
#pragma unroll
    for (int c = 0; c < DP4; c++) v[c] = rows[q * DP4 + c];
  }
  __device__ __forceinline__ float dist2(const float4 *__restrict__ r, int) const {
    return dist2_rows<DP4>(v, r);
  }
  // Member row (already in registers): distance and (IDXROW) the index
  // stored in the row's last pad float.
  __device__ __forceinline__ float dist2_member(const float4 (&row)[DP4],
                                                int32_t *idx) const {
    float acc = 0.0f;
#pragma unroll
    for (int c = 0; c < DP4; c++) {
      const float4 s = row[c];
      float t;
      t = __fsub_rn(v[c].x, s.x); acc = __fmaf_rn(t, t, acc);
      t = __fsub_rn(v[c].y, s.y); acc = __fmaf_rn(t, t, acc);
      t = __fsub_rn(v[c].z, s.z); acc = __fmaf_rn(t, t, acc);
      if (IDXROW && c == DP4 - 1) {
        *idx = __float_as_int(s.w);
      } else {
        t = __fsub_rn(v[c].w, s.w); acc = __fmaf_rn(t, t, acc);
      }
    }
    return acc;
  }
};

// Runtime width: the query row lives in the warp's shared-memory slot.
template <bool IDXROW>
struct QueryRow<0, IDXROW> {
  const float4 *v;
  __device__ __forceinline__ void load(const float4 *__restrict__ rows, int64_t q, int dp4,
                                       float4 *slot) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    for (int c = lane; c < dp4; c += 32) slot[c] = rows[q * dp4 + c];
    __syncwarp();
    v = slot;
  }
  __device__ __forceinline__ float dist2(const float4 *__restrict__ r, int dp4) const {
    return dist2_rows_rt(v, r, dp4);
  }
};

// Resident warps per SM the register allocation must allow (compile-time
// tuning knobs): the scan is latency-bound, so occupancy matters; rows of
// more than 8 floats keep the query in registers and get the lower target.
#ifndef KNN_TARGET_WARPS
#define KNN_TARGET_WARPS 32
#endif
#ifndef KNN_TARGET_WARPS_WIDE
#define KNN_TARGET_WARPS_WIDE 16
#endif
// Load a small member row together with its band distance (before the band
// test) so both loads are in flight at once.
#ifndef KNN_EAGER_ROWS
#define KNN_EAGER_ROWS 1
#endif

// Traversal choices (compile-time): visit a chunk's clusters nearest d(q,Rs)
// first, and walk each band outward from d(s,Rs) ~ d(q,Rs).
#ifndef KNN_ORDER_BY_D
#define KNN_ORDER_BY_D 1
#endif
#ifndef KNN_WALK_OUTWARD
#define KNN_WALK_OUTWARD 0
#endif
// Visits take a cluster's bounds and member range from the lanes that tested
// it (loaded once per batch of 32 candidate clusters) and start the band
// walk from the coarse member search (1); or reload them per visit and
// search to the exact band edge (0).
#ifndef KNN_VISIT_META
#define KNN_VISIT_META 1
#endif

#ifndef KNN_INDEX32
#define KNN_INDEX32 1
#endif

// The thread-per-query scan keeps its statistics counters in shared memory
// (1) or in registers (0).
#ifndef KNN_TSCAN_SMEM_STATS
#define KNN_TSCAN_SMEM_STATS 1
#endif
// The query's slot, row and cluster wait out the walk in shared memory (1)
// or in registers (0).
#ifndef KNN_SIDE_WORDS
#define KNN_SIDE_WORDS 1
#endif

// Largest k kept in a register list (one key per lane): up to 24, so that
// 8 of the 32 slots or more hold the FP32 band behind the k-th; larger k use
// the shared-memory candidate set.
#ifndef KNN_REG_TOPK_MAX_K
#define KNN_REG_TOPK_MAX_K 24
#endif

template <int L>
using TopKFor = std::conditional_t<(L <= 32), RegTopK<L / 32>, SelectTopK<L>>;

// Rows of more than 8 floats keep 4+ float4 of the query in registers: those
// kernels get the lower occupancy target instead of spilling.
template <int DP4, int WARPS>
constexpr int scan_min_blocks() {
  return ((DP4 == 0 || DP4 >= 4) ? KNN_TARGET_WARPS_WIDE : KNN_TARGET_WARPS) / WARPS;
}

template <int DP4, bool IDXROW, int L, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (scan_min_blocks<DP4, WARPS>()))
    scan_kernel(const ScanArgs a) {
  using TK = TopKFor<L>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int dp4 = DP4 > 0 ? DP4 : a.dp4;
  uint64_t *keys_base = reinterpret_cast<uint64_t *>(smem_raw);
  float4 *qslot = reinterpret_cast<float4 *>(keys_base + (size_t)WARPS * TK::kSmemKeys) +
                  (size_t)w * (DP4 > 0 ? 0 : a.dp4);
  TK tk;
  tk.init(keys_base + (size_t)w * TK::kSmemKeys);
  tk.k = a.k;
  const float tol = bound_tol(a.d);
  unsigned evals = 0;
  constexpr bool kWideRows = DP4 == 0 || DP4 >= 4;
  // small rows: load the member row together with its band distance
  constexpr bool kEagerRow = KNN_EAGER_ROWS && (DP4 > 0 && DP4 <= 2);
  // statistics: per-lane 32-bit counts folded once per query into per-block
  // shared counters, added to the global ones at exit
  __shared__ unsigned long long blk_ctr[kScanCounters];
  if (threadIdx.x < kScanCounters) blk_ctr[threadIdx.x] = 0;
  if (lane < kStatWords) tk.stat()[lane] = 0;
  __syncthreads();

  for (;;) {
    long long slot = 0;
    if (lane == 0) slot = (long long)atomicAdd(a.work_counter, 1ull);
    slot = __shfl_sync(kFull, slot, 0);
    if (a.slot_list) {
      if (slot >= (long long)*a.slot_count) break;
      slot = a.slot_list[slot];
    } else if (slot >= a.m) {
      break;
    } else {
      slot += a.slot_base;
    }
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
#if KNN_SIDE_WORDS
    if (lane == 0) {
      unsigned *sw = tk.stat();
      sw[kSideSlot] = (unsigned)slot;
      sw[kSideQuery] = (unsigned)q;
      sw[kSideCluster] = (unsigned)qc;
      sw[kSideDq] = a.qkeys ? (uint32_t)a.qkeys[slot] : 0x7f800000u;  // +inf: no exit
    }
#endif
    QueryRow<DP4, IDXROW> qr;
    qr.load(a.qrows, q, dp4, qslot);
    tk.reset(query_theta0(a, slot, qc, tol), lane);

    // one band step: lane's member p of the cluster at `start`, kept when
    // its distance to the representative lies in [lo_v, hi_v]
    auto step = [&](int start, int p, bool valid, float lo_v, float hi_v) -> float {
#if KNN_INDEX32
      // row indices fit 32 bits (the result indices are int32): unsigned
      // offsets make every address one wide multiply-add
      const unsigned gp = (unsigned)(start + p);
#else
      const int64_t gp = (int64_t)start + p;
#endif
      float dsv = 0.0f, v = 0.0f;
      int32_t idx = 0;
      bool inb;
      if constexpr (kEagerRow) {
        // small rows: issue the row load together with the band distance
        float4 row[DP4];
        if (valid) {
#pragma unroll
          for (int c = 0; c < DP4; c++) row[c] = a.srows[(size_t)gp * DP4 + c];
          dsv = a.sdist[gp];
        }
        inb = valid && dsv >= lo_v && dsv <= hi_v;
        if (inb) v = qr.dist2_member(row, &idx);
      } else if constexpr (DP4 > 0) {
        dsv = valid ? a.sdist[gp] : 0.0f;
        inb = valid && dsv >= lo_v && dsv <= hi_v;
        if (inb) {
          float4 row[DP4];
#pragma unroll
          for (int c = 0; c < DP4; c++) row[c] = a.srows[(size_t)gp * DP4 + c];
          v = qr.dist2_member(row, &idx);
        }
      } else {
        dsv = valid ? a.sdist[gp] : 0.0f;
        inb = valid && dsv >= lo_v && dsv <= hi_v;
        if (inb) v = qr.dist2(a.srows + (size_t)gp * dp4, dp4);
      }
      bool pass = false;
      if (inb) {
        evals++;
        pass = v <= tk.thr_d2;
        if (!IDXROW && pass) idx = a.sidx[gp];
      }
      topk_offer(tk, pass, v, idx, lane, a.d);
      return dsv;
    };

    const int nr = a.rlen[qc];
    const int32_t *rl = a.rlist + (a.rl_base ? a.rl_base[qc] : (int64_t)qc * a.Rs);
    for (int base = 0; base < nr; base += 32) {
#if KNN_CHUNK_EXIT && KNN_SIDE_WORDS
      // the rest of the list is prunable when even its nearest cluster
      // (the list is ascending in d(Rq,Rs)) lies beyond theta for the
      // largest remaining radius: d(q,Rs) - cmax >= d(Rq,Rs) - d(q,Rq) -
      // max cmax; the filter's own test, with twice its rounding margin.
      // Rows of 16 floats or more (d = 32: scan 6.14 -> 5.61 ms, d = 128:
      // 14.88 -> 13.42 ms); on the k = 200, d = 3 self-join the test cost
      // more than it saved (3.82 -> 3.87 ms)
      if (kWideRows && a.clb) {
        const unsigned *sw = tk.stat();
        const float2 cb = a.clb[(size_t)sw[kSideCluster] * a.clb_stride + (base >> 5)];
        const float dqv = __uint_as_float(sw[kSideDq]), th = tk.theta;
        if (cb.x - dqv - cb.y > th + 2.0f * tol * (cb.x + dqv + cb.y + th)) {
          tk.count(kStatPruned, (unsigned)(nr - base), lane);
          break;
        }
      }
#endif
      const int j = base + lane;
      int rs = 0;
      float D = 0.0f;
      bool alive = false;
#if KNN_VISIT_META
      float cmx = 0.0f, cmn = 0.0f;
      int cst = 0, cnn = 0;
#endif
      if (j < nr) {
        rs = rl[j];
        D = sqrtf(qr.dist2(a.sreps + (int64_t)rs * dp4, dp4));
        const float th = tk.theta;
        const float slack = tol * (2.0f * D + 2.0f * th);
#if KNN_VISIT_META
        cmx = a.cmax[rs];
        cmn = a.cmin[rs];
        alive = !(D - cmx > th + slack) && !(D + th + slack < cmn);
        if (alive) {
          cst = a.soff[rs];
          cnn = a.soff[rs + 1] - cst;
        }
#else
        alive = !(D - a.cmax[rs] > th + slack) && !(D + th + slack < a.cmin[rs]);
#endif
      }
      // visit this chunk's surviving clusters: in list order (by rep-rep
      // distance) or, with KNN_ORDER_BY_D, nearest d(q, Rs) first
      unsigned amask = __ballot_sync(kFull, alive);
      tk.count(kStatPruned, (unsigned)(min(32, nr - base) - __popc(amask)), lane);
      if (amask == 0) continue;  // warp-uniform: nothing to visit in this batch
      const int nalive = __popc(amask);
      float dkey = alive ? D : __int_as_float(0x7f800000);
      // Visit order: nearest d(q, Rs) first.  Narrow rows sort the batch once
      // (bitonic network over the 32 lanes, ties to the lower lane: less work
      // per visited cluster); wider rows pick the nearest remaining cluster
      // by a warp arg-min per visit (measured faster there).
      constexpr bool kSortBatch = KNN_ORDER_BY_D != 0 && DP4 >= 1 && DP4 <= 2;
      float sv = dkey;
      int sl = lane;
      if (kSortBatch && nalive > 1) {  // a single survivor needs no order
#pragma unroll
        for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
          for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const float ov = __shfl_xor_sync(kFull, sv, stride);
            const int ol = __shfl_xor_sync(kFull, sl, stride);
            const bool other_less = ov < sv || (ov == sv && ol < sl);
            const bool keep_min = ((lane & stride) == 0) == ((lane & size) == 0);
            if (other_less == keep_min) {
              sv = ov;
              sl = ol;
            }
          }
        }
      }
      for (int rank = 0; rank < nalive; rank++) {
        int src;
        if constexpr (kSortBatch) {
          src = nalive > 1 ? __shfl_sync(kFull, sl, rank) : __ffs(amask) - 1;
        } else {
          src = __ffs(amask) - 1;
#if KNN_ORDER_BY_D
          if (amask & (amask - 1)) {
            float mv = dkey;
            int ml = lane;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              const float ov = __shfl_xor_sync(kFull, mv, o);
              const int ol = __shfl_xor_sync(kFull, ml, o);
              if (ov < mv || (ov == mv && ol < ml)) {
                mv = ov;
                ml = ol;
              }
            }
            src = ml;
          }
          if (lane == src) dkey = __int_as_float(0x7f800000);
#endif
          amask &= ~(1u << src);
        }
        const float Dc = __shfl_sync(kFull, D, src);
#if KNN_VISIT_META
        const float cmax_c = __shfl_sync(kFull, cmx, src);
        const float cmin_c = __shfl_sync(kFull, cmn, src);
#else
        const int c = __shfl_sync(kFull, rs, src);
        const float cmax_c = a.cmax[c], cmin_c = a.cmin[c];
#endif
        float th = tk.theta;
        float slack = tol * (2.0f * Dc + 2.0f * th);
        if (Dc - cmax_c > th + slack || Dc + th + slack < cmin_c) {
          tk.count(kStatPruned, 1, lane);
          continue;
        }
        tk.count(kStatVisited, 1, lane);
#if KNN_VISIT_META
        const int start = __shfl_sync(kFull, cst, src);
        const int n_c = __shfl_sync(kFull, cnn, src);
#else
        const int start = a.soff[c];
        const int n_c = a.soff[c + 1] - start;
#endif
#if KNN_WALK_OUTWARD
        // members below `mid` have d(s,Rs) < Dc, from `mid` on >= Dc; walk
        // outward from there, alternately up and down
        const int mid = warp_lower_bound(a.sdist + start, n_c, Dc, lane);
        int up = mid, dn = mid;
        bool go_up = up < n_c, go_dn = dn > 0;
        while (go_up || go_dn) {
          if (go_up) {
            th = tk.theta;
            slack = tol * (2.0f * Dc + 2.0f * th);
            const float hi_v = Dc + th + slack;
            const int p = up + lane;
            const bool valid = p < n_c;
            const float dsv = step(start, p, valid, -1.0f, hi_v);
            const bool past = !valid || dsv > hi_v;
            up += 32;
            if (__shfl_sync(kFull, past, 31) || up >= n_c) go_up = false;
          }
          if (go_dn) {
            th = tk.theta;
            slack = tol * (2.0f * Dc + 2.0f * th);
            const float lo_v = Dc - th - slack;
            const int p = dn - 32 + lane;
            const bool valid = p >= 0;
            const float dsv = step(start, p, valid, lo_v, __int_as_float(0x7f800000));
            const bool past = !valid || dsv < lo_v;
            dn -= 32;
            if (__shfl_sync(kFull, past, 0) || dn <= 0) go_dn = false;
          }
        }
#else
        // one direction: from the lower band edge up (no search when the band
        // starts below the cluster's nearest member)
        const float lo_edge = Dc - th - slack;
#if KNN_VISIT_META
        const int lo = lo_edge <= cmin_c ? 0 : warp_lower_bound_coarse(a.sdist + start, n_c, lo_edge, lane);
#else
        const int lo = lo_edge <= cmin_c ? 0 : warp_lower_bound(a.sdist + start, n_c, lo_edge, lane);
#endif
        for (int p0 = lo; p0 < n_c; p0 += 32) {
          th = tk.theta;
          slack = tol * (2.0f * Dc + 2.0f * th);
          const float hi_v = Dc + th + slack, lo_v = Dc - th - slack;
          const int p = p0 + lane;
          const bool valid = p < n_c;
          const float dsv = step(start, p, valid, lo_v, hi_v);
          const bool past = !valid || dsv > hi_v;
          if (__shfl_sync(kFull, past, 31)) break;
        }
#endif
      }
    }
    tk.finish(lane, a.d);
#if KNN_SIDE_WORDS
    __syncwarp();
    {
      const unsigned *sw = tk.stat();
      const int32_t e_slot = (int32_t)sw[kSideSlot];
      const int64_t e_q = (int64_t)sw[kSideQuery];
      const int e_qc = (int)sw[kSideCluster];
      tk.count(kStatChecked, emit_query(tk, a, e_slot, e_q, e_qc, lane), lane);
    }
#else
    tk.count(kStatChecked, emit_query(tk, a, (int32_t)slot, q, qc, lane), lane);
#endif
    __syncwarp();
    if (a.counters) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(kFull, evals, o);
      if (lane == 0) {
        const unsigned *st = tk.stat();
        atomicAdd(&blk_ctr[0], (unsigned long long)evals);
        atomicAdd(&blk_ctr[1], (unsigned long long)st[kStatVisited]);
        atomicAdd(&blk_ctr[2], (unsigned long long)st[kStatPruned]);
        atomicAdd(&blk_ctr[3], (unsigned long long)st[kStatPushed]);
        atomicAdd(&blk_ctr[4], (unsigned long long)st[kStatMerges]);
        atomicAdd(&blk_ctr[5], (unsigned long long)st[kStatChecked]);
      }
    }
    __syncwarp();
    if (lane < kStatWords) tk.stat()[lane] = 0;
    evals = 0;
  }
  __syncthreads();
  if (a.counters && threadIdx.x < kScanCounters)
    atomicAdd(a.counters + threadIdx.x, blk_ctr[threadIdx.x]);
}

template <int DP4, bool IDXROW, int L, int WARPS>
static int launch_scan_t(const ScanArgs &a, int num_sms, cudaStream_t s) {
  using TK = TopKFor<L>;
  const size_t smem = (size_t)WARPS * TK::kSmemKeys * sizeof(uint64_t) +
                      (DP4 > 0 ? 0 : (size_t)WARPS * a.dp4 * sizeof(float4));
  auto kern = scan_kernel<DP4, IDXROW, L, WARPS>;
  if (smem > 48 * 1024)
    KNN_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  int per_sm = 0;
  KNN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t want = (a.m + WARPS - 1) / WARPS;
  int64_t grid = (int64_t)num_sms * per_sm;
  if (grid > want) grid = want;
  if (grid < 1) grid = 1;
  kern<<<(int)grid, WARPS * 32, smem, s>>>(a);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

template <int DP4, bool IDXROW>
static int launch_scan_l(const ScanArgs &a, int num_sms, cudaStream_t s) {
  if (a.k <= KNN_REG_TOPK_MAX_K) return launch_scan_t<DP4, IDXROW, 32, 8>(a, num_sms, s);
  if (a.k <= 64) return launch_scan_t<DP4, IDXROW, 64, 8>(a, num_sms, s);
  if (a.k <= 128) return launch_scan_t<DP4, IDXROW, 128, 8>(a, num_sms, s);
  if (a.k <= 256) return launch_scan_t<DP4, IDXROW, 256, 8>(a, num_sms, s);
  if (a.k <= 512) return launch_scan_t<DP4, IDXROW, 512, 4>(a, num_sms, s);
  return launch_scan_t<DP4, IDXROW, 1024, 4>(a, num_sms, s);
}

// ---------------------------------------------------------------------------
// Thread-per-query scan for small k (k <= 32) and narrow rows (d <= 8).  With
// few distances per query (k = 16 on a surface: ~200) the warp-per-query
// scan spends most of its instructions on per-query and per-cluster overhead
// (lane-parallel cluster tests, nearest-first ordering, 32-ary band search,
// list merges) for bands that fill few lanes.  Here every thread walks its own
// query, in the same order of the same candidate list, with the same pruning
// tests and the same FP32 keys, keeping its K best keys sorted in registers
// (K = pow2 >= k; the K-th key is the pruning bound, so for k < K the bound is
// looser but the first k keys are still the k nearest).  The 32 queries of a
// warp are consecutive slots, mostly of one query cluster, so they walk
// similar lists.
// ---------------------------------------------------------------------------
template <int K>
struct ThreadTopK {
  uint64_t key[K];  // ascending; kKeyMax = empty
  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int j = 0; j < K; j++) key[j] = kKeyMax;
  }
  // inserts v, which must be smaller than key[K-1]
  __device__ __forceinline__ void insert(uint64_t v) {
#pragma unroll
    for (int j = K - 1; j > 0; j--) {
      const uint64_t prev = key[j - 1];
      key[j] = prev > v ? prev : (key[j] > v ? v : key[j]);
    }
    key[0] = key[0] > v ? v : key[0];
  }
};

// 4 blocks per SM (64 registers; 71 unbounded gave 3): C4 79.3 -> 76.5 ms.
// Loading member p + 1 while member p is evaluated measured slower.
//
// FP64 boundary: the pruning bound is band_hi of the K-th key, so every point
// inside the final k-th's FP32 band is evaluated; one that does not fit the
// list sets `lost`.  A query whose band reaches behind its k-th (a key inside
// it was lost, or the list holds one after the k-th) goes to the band kernel,
// which re-decides the band in FP64; on data without near-ties at the k-th
// that is a small fraction of the queries, and FP64 code stays out of this
// register-bound kernel.
template <int DP4, bool IDXROW, int K>
__global__ void __launch_bounds__(256, 4)
    thread_scan_kernel(const ScanArgs a) {
  __shared__ unsigned long long blk_ctr[kScanCounters];
  if (threadIdx.x < kScanCounters) blk_ctr[threadIdx.x] = 0;
  __syncthreads();
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nslots = a.slot_list ? (int64_t)*a.slot_count : a.m;
#if KNN_TSCAN_SMEM_STATS
  // visited, pruned, pushed of this thread's query in shared memory (stride
  // 3 words: no bank conflicts), out of the walk's registers
  __shared__ unsigned tstat[3 * 256];
  unsigned *ts = tstat + 3 * threadIdx.x;
  ts[0] = ts[1] = ts[2] = 0;
  unsigned evals = 0;
#else
  unsigned evals = 0, visited = 0, pruned = 0, pushed = 0;
#endif
  if (t < nslots) {
    const int64_t slot = a.slot_list ? (int64_t)a.slot_list[t] : a.slot_base + t;
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
    const int d = a.d;
    const float tol = bound_tol(d);
    QueryRow<DP4, IDXROW> qr;
    qr.load(a.qrows, q, DP4, nullptr);
    ThreadTopK<K> tk;
    tk.reset();
    float theta = query_theta0(a, slot, qc, tol);
    float lost = __int_as_float(0x7f800000);
    // admits every d^2 <= theta0^2, whatever the index
    const uint64_t thr0 = ((uint64_t)__float_as_uint(theta * theta) << 32) | 0xffffffffull;
    const int nr = a.rlen[qc];
    const int32_t *rl = a.rlist + (a.rl_base ? a.rl_base[qc] : (int64_t)qc * a.Rs);
    for (int j = 0; j < nr; j++) {
      const int c = rl[j];
      const float D = sqrtf(qr.dist2(a.sreps + (int64_t)c * DP4, DP4));
      float slack = tol * (2.0f * D + 2.0f * theta);
      const float cmin = a.cmin[c];
      if (D - a.cmax[c] > theta + slack || D + theta + slack < cmin) {
#if KNN_TSCAN_SMEM_STATS
        ts[1]++;
#else
        pruned++;
#endif
        continue;
      }
#if KNN_TSCAN_SMEM_STATS
      ts[0]++;
#else
      visited++;
#endif
      const int start = a.soff[c], n_c = a.soff[c + 1] - start;
      const float *sd = a.sdist + start;
      // first member of the band [D - theta, D + theta] (with slack)
      const float lo_edge = D - theta - slack;
      int p = 0;
      if (lo_edge > cmin) {
        int hi = n_c;
        while (p < hi) {
          const int md = (p + hi) >> 1;
          if (sd[md] < lo_edge) p = md + 1;
          else hi = md;
        }
      }
      for (; p < n_c; p++) {
        if (sd[p] > D + theta + slack) break;
        float4 row[DP4];
#pragma unroll
        for (int cc = 0; cc < DP4; cc++) row[cc] = a.srows[(int64_t)(start + p) * DP4 + cc];
        int32_t idx = 0;
        const float v = qr.dist2_member(row, &idx);
        evals++;
        if (!IDXROW) idx = a.sidx[start + p];
        const uint64_t key = make_key(v, idx);
        if (key < thr0) {
          if (key < tk.key[K - 1]) {
            lost = fminf(lost, key_d2(tk.key[K - 1]));  // NaN (empty) is ignored
            tk.insert(key);
#if KNN_TSCAN_SMEM_STATS
            ts[2]++;
#else
            pushed++;
#endif
            if (tk.key[K - 1] != kKeyMax) {
              theta = sqrtf(band_hi(key_d2(tk.key[K - 1]), d));
              slack = tol * (2.0f * D + 2.0f * theta);
            }
          } else {
            lost = fminf(lost, v);
          }
        }
      }
    }
    // the k-th key, the key behind it, and the FP32 band around the k-th
    // (selected by masks: a compare-and-select on the runtime k turns the
    // list into an indexed local-memory array)
    uint64_t kth = 0, next = 0;
#pragma unroll
    for (int j = 0; j < K; j++) {
      kth |= tk.key[j] & (0ull - (uint64_t)(j == a.k - 1));
      next |= tk.key[j] & (0ull - (uint64_t)(j == a.k));
    }
    if (a.k >= K) next = kKeyMax;
    bool defer = false;
    int nlo = 0;
    const float Dk = key_d2(kth);
    if (kth != kKeyMax && !fp32_exact(a)) {
      const float hi = band_hi(Dk, d);
      // a band key was dropped, or one sits behind the k-th (NaN: none)
      defer = lost <= hi || key_d2(next) <= hi;
      if (defer) {
        const float lo = band_lo(Dk, d);
#pragma unroll
        for (int j = 0; j < K; j++) nlo += key_d2(tk.key[j]) < lo;
      }
    }
    int32_t *oi = a.out_idx + q * a.k;
    float *od = a.out_dist + q * a.k;
    const int32_t base = a.qc_ref_base ? (int32_t)a.qc_ref_base[qc] : 0;
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (j < a.k) {
        const uint64_t key = tk.key[j];
        const bool none = key == kKeyMax;
        oi[j] = none ? -1 : key_idx(key) - base;
        const float d2 = key_d2(key);
        od[j] = none ? __int_as_float(0x7f800000) : (a.squared ? d2 : sqrtf(d2));
      }
    }
    if (defer) {
      // the band kernel settles the boundary: it reads the number of keys
      // below the band and the k-th value from the last slot
      oi[a.k - 1] = nlo;
      od[a.k - 1] = Dk;
      a.unres_slot[atomicAdd(a.unres_count, 1u)] = (int32_t)slot;
    }
  }
  if (a.counters) {
#if KNN_TSCAN_SMEM_STATS
    unsigned visited = ts[0], pruned = ts[1], pushed = ts[2];
#endif
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      evals += __shfl_xor_sync(kFull, evals, o);
      visited += __shfl_xor_sync(kFull, visited, o);
      pruned += __shfl_xor_sync(kFull, pruned, o);
      pushed += __shfl_xor_sync(kFull, pushed, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&blk_ctr[0], (unsigned long long)evals);
      atomicAdd(&blk_ctr[1], (unsigned long long)visited);
      atomicAdd(&blk_ctr[2], (unsigned long long)pruned);
      atomicAdd(&blk_ctr[3], (unsigned long long)pushed);
    }
    __syncthreads();
    if (threadIdx.x < kScanCounters) atomicAdd(a.counters + threadIdx.x, blk_ctr[threadIdx.x]);
  }
}

template <int DP4, bool IDXROW>
static int launch_thread_scan(const ScanArgs &a, cudaStream_t s) {
  const int blocks = (int)((a.m + 255) / 256);
  auto go = [&](auto kern) -> int {
    kern<<<blocks, 256, 0, s>>>(a);
    KNN_LAUNCH_CHECK();
    return KNN_OK;
  };
  if (a.k <= 1) return go(thread_scan_kernel<DP4, IDXROW, 1>);
  if (a.k <= 2) return go(thread_scan_kernel<DP4, IDXROW, 2>);
  if (a.k <= 4) return go(thread_scan_kernel<DP4, IDXROW, 4>);
  if (a.k <= 8) return go(thread_scan_kernel<DP4, IDXROW, 8>);
  if (a.k <= 16) return go(thread_scan_kernel<DP4, IDXROW, 16>);
  return go(thread_scan_kernel<DP4, IDXROW, 32>);
}

// ---------------------------------------------------------------------------
// Band kernel: the k-th boundary of the queries the scan kernels could not
// settle (a key of the final band was dropped for lack of room, or the
// thread scan's list holds one behind the k-th).  One block per query, over
// the same candidate list: every point whose FP32 d^2 -- computed with the
// scan's own arithmetic, so the values are the same -- lies inside the band
// band_lo(Dk) .. band_hi(Dk) of the k-th is found again, and the band's
// need = k - nlo best by (FP64 d^2, index) are kept in a shared-memory set
// that is sorted and cut back to `need` whenever it fills, so any number of
// ties fits.  They are written, in FP32 key order, behind the nlo keys below
// the band that the scan already wrote.  The scan left nlo and Dk in the
// query's last output slot.
// ---------------------------------------------------------------------------
constexpr int kBandThreads = 128;
constexpr int kBandCap = 2048;  // >= KNN_MAX_K + kBandThreads: room after a cut

struct BandEntry {
  unsigned long long d64;  // FP64 d^2 bits (non-negative: they order like the values)
  unsigned long long key;  // FP32 (d^2, index) key
};

__device__ __forceinline__ bool band_entry_less(const BandEntry &x, const BandEntry &y) {
  return x.d64 < y.d64 || (x.d64 == y.d64 && (uint32_t)x.key < (uint32_t)y.key);
}

// Ascending bitonic sort of e[0..P) (P a power of two) by the block, by
// (FP64 d^2, index) or by the FP32 key.
template <bool BY_KEY>
__device__ void band_sort(BandEntry *e, int P) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const BandEntry x = e[i], y = e[j];
        const bool gt = BY_KEY ? x.key > y.key : band_entry_less(y, x);
        if (gt == up) {
          e[i] = y;
          e[j] = x;
        }
      }
      __syncthreads();
    }
  }
}

// Cuts the set e[0..*cnt) back to its `need` smallest by (FP64 d^2, index);
// *thr becomes the need-th (the admission bound) once that many are in.
__device__ void band_cut(BandEntry *e, int *cnt, BandEntry *thr, int need) {
  const int c = *cnt;  // read by every thread before the barrier below
  int P = 1;
  while (P < c) P <<= 1;
  for (int i = c + threadIdx.x; i < P; i += blockDim.x) e[i] = BandEntry{~0ull, ~0ull};
  __syncthreads();
  band_sort<false>(e, P);
  if (threadIdx.x == 0) {
    const int kept = c < need ? c : need;
    *cnt = kept;
    if (kept == need) *thr = e[need - 1];
  }
  __syncthreads();
}

// FP32 squared distance over the first d coordinates, dimension order, fma:
// the scan kernels' value for the same pair (their padded coordinates add
// exact zeros).
__device__ __forceinline__ float band_dist2(const float *__restrict__ q,
                                            const float *__restrict__ r, int d) {
  float acc = 0.0f;
  for (int c = 0; c < d; c++) {
    const float t = __fsub_rn(q[c], r[c]);
    acc = __fmaf_rn(t, t, acc);
  }
  return acc;
}

__global__ void __launch_bounds__(kBandThreads) band_resolve_kernel(const ScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BandEntry *ent = reinterpret_cast<BandEntry *>(smem_raw);
  float *qv = reinterpret_cast<float *>(ent + kBandCap);  // 4 * dp4 floats
  __shared__ int s_cnt;
  __shared__ BandEntry s_thr;
  const int tid = threadIdx.x, k = a.k, d = a.d, dp4 = a.dp4;
  const float tol = bound_tol(d);
  const unsigned total = *a.unres_count;
  unsigned long long evals = 0;
  for (unsigned u = blockIdx.x; u < total; u += gridDim.x) {
    const int32_t slot = a.unres_slot[u];
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
    int32_t *oi = a.out_idx + q * k;
    float *od = a.out_dist + q * k;
    __syncthreads();  // the previous query is done with the shared state
    const int nlo = oi[k - 1];
    const float Dk = od[k - 1];
    const int need = k - nlo;
    const float lo = band_lo(Dk, d), hi = band_hi(Dk, d), th = sqrtf(hi);
    for (int c = tid; c < 4 * dp4; c += kBandThreads)
      qv[c] = reinterpret_cast<const float *>(a.qrows + q * dp4)[c];
    if (tid == 0) {
      s_cnt = 0;
      s_thr = BandEntry{~0ull, ~0ull};
    }
    __syncthreads();
    const int nr = a.rlen[qc];
    const int32_t *rl = a.rlist + (a.rl_base ? a.rl_base[qc] : (int64_t)qc * a.Rs);
    for (int j = 0; j < nr; j++) {  // block-uniform
      const int c = rl[j];
      const float D =
          sqrtf(band_dist2(qv, reinterpret_cast<const float *>(a.sreps + (int64_t)c * dp4), d));
      const float slack = tol * (2.0f * D + 2.0f * th);
      if (D - a.cmax[c] > th + slack || D + th + slack < a.cmin[c]) continue;
      const int start = a.soff[c], n_c = a.soff[c + 1] - start;
      const float lo_e = D - th - slack, hi_e = D + th + slack;
      int p0 = 0, p1 = n_c;  // first member with d(s, Rc) >= lo_e
      while (p0 < p1) {
        const int md = (p0 + p1) >> 1;
        if (a.sdist[start + md] < lo_e) p0 = md + 1;
        else p1 = md;
      }
      for (int c0 = p0; c0 < n_c; c0 += kBandThreads) {  // block-uniform
        const int p = c0 + tid;
        bool past = p >= n_c;
        if (!past) {
          const int64_t gp = (int64_t)start + p;
          if (a.sdist[gp] > hi_e) {
            past = true;
          } else {
            const float v =
                band_dist2(qv, reinterpret_cast<const float *>(a.srows + gp * dp4), d);
            if (v >= lo && v <= hi) {
              const int32_t id = a.sidx[gp];
              const double w =
                  dist2_f64(qv, reinterpret_cast<const float *>(a.rrows + (int64_t)id * dp4), d);
              evals++;
              const BandEntry e{(unsigned long long)__double_as_longlong(w), make_key(v, id)};
              if (band_entry_less(e, s_thr)) ent[atomicAdd(&s_cnt, 1)] = e;
            }
          }
        }
        const int any_past = __syncthreads_or(past);
        if (s_cnt > kBandCap - kBandThreads) band_cut(ent, &s_cnt, &s_thr, need);
        if (any_past) break;
      }
    }
    band_cut(ent, &s_cnt, &s_thr, need);
    // the band's share of the result, in FP32 key order
    const int got = s_cnt;  // == need: the scan's own band keys are all found again
    int P = 1;
    while (P < got) P <<= 1;
    for (int i = got + tid; i < P; i += kBandThreads) ent[i] = BandEntry{~0ull, ~0ull};
    __syncthreads();
    band_sort<true>(ent, P);
    const int32_t base = a.qc_ref_base ? (int32_t)a.qc_ref_base[qc] : 0;
    for (int t = tid; t < need; t += kBandThreads) {
      const uint64_t key = t < got ? ent[t].key : kKeyMax;
      const bool none = key == kKeyMax;
      oi[nlo + t] = none ? -1 : key_idx(key) - base;
      od[nlo + t] =
          none ? __int_as_float(0x7f800000) : (a.squared ? key_d2(key) : sqrtf(key_d2(key)));
    }
  }
  if (a.counters) {
    for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(kFull, evals, o);
    if ((tid & 31) == 0 && evals) atomicAdd(a.counters + 5, evals);
    if (blockIdx.x == 0 && tid == 0) atomicAdd(a.counters + 6, (unsigned long long)total);
  }
}

static int launch_band_resolve(const ScanArgs &a, int num_sms, cudaStream_t s) {
  const size_t smem = kBandCap * sizeof(BandEntry) + (size_t)a.dp4 * sizeof(float4);
  if (smem > 48 * 1024)
    KNN_CUDA_TRY(cudaFuncSetAttribute(band_resolve_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // a persistent grid over the list, whose length only the device knows
  // (an empty list costs one launch that returns at once)
  band_resolve_kernel<<<2 * num_sms, kBandThreads, smem, s>>>(a);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

#ifndef KNN_THREAD_SCAN_MAX_K
#define KNN_THREAD_SCAN_MAX_K 32
#endif

static int launch_scan_kernels(const ScanArgs &a, int num_sms, cudaStream_t s);

// The scan of one batch of query slots, then the band kernel for the queries
// whose k-th boundary the scan left open.
int launch_scan(const ScanArgs &a, int num_sms, cudaStream_t s) {
  if (a.m == 0) return KNN_OK;
  if (!a.rrows || !a.unres_slot || !a.unres_count) {
    set_error("scan: the FP64 boundary buffers are missing");
    return KNN_EINTERNAL;
  }
  KNN_CUDA_TRY(cudaMemsetAsync(a.unres_count, 0, sizeof(unsigned), s));
  const int rc = launch_scan_kernels(a, num_sms, s);
  if (rc != KNN_OK) return rc;
  return launch_band_resolve(a, num_sms, s);
}

static int launch_scan_kernels(const ScanArgs &a, int num_sms, cudaStream_t s) {
  // thread per query: small k, rows of at most 8 floats, and short bands (at
  // most 128 points per cluster on average).  Measured: 4,096 surface clouds
  // (~70-100 points per cluster, k = 16) 143 -> 67 ms; a dense 3-D set with
  // ~300 points per cluster at k = 32 2.7 -> 4.3 ms (slower); d = 16 and 32
  // slower too.
  const bool short_bands = a.n_ref > 0 && a.Rs > 0 && a.n_ref <= 128 * (int64_t)a.Rs;
  if (a.k <= KNN_THREAD_SCAN_MAX_K && short_bands && (a.dp4_tmpl == 1 || a.dp4_tmpl == 2)) {
    if (a.dp4_tmpl == 1)
      return a.idx_in_row ? launch_thread_scan<1, true>(a, s) : launch_thread_scan<1, false>(a, s);
    return a.idx_in_row ? launch_thread_scan<2, true>(a, s) : launch_thread_scan<2, false>(a, s);
  }
  switch (a.dp4_tmpl) {
    case 1: return a.idx_in_row ? launch_scan_l<1, true>(a, num_sms, s)
                                : launch_scan_l<1, false>(a, num_sms, s);
    case 2: return a.idx_in_row ? launch_scan_l<2, true>(a, num_sms, s)
                                : launch_scan_l<2, false>(a, num_sms, s);
    case 4: return a.idx_in_row ? launch_scan_l<4, true>(a, num_sms, s)
                                : launch_scan_l<4, false>(a, num_sms, s);
    case 8: return a.idx_in_row ? launch_scan_l<8, true>(a, num_sms, s)
                                : launch_scan_l<8, false>(a, num_sms, s);
    default: return launch_scan_l<0, false>(a, num_sms, s);
  }
}

}  // namespace knnsweet
