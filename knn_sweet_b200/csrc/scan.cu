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
//     contiguous band around the member whose d(s,Rs) is closest to D.  A
//     warp-wide 32-ary search finds that member; the warp then walks outward,
//     32 members per step, alternately up and down, with coalesced row loads,
//     and stops in each direction at the first step that leaves the band
//     (re-evaluated with the current theta).
//   - Exact FP32 distances go through the warp top-k: candidates whose
//     (d^2, index) key beats the current k-th key are appended to a
//     shared-memory buffer; a full buffer is sorted and merged into the sorted
//     list of the k best, after which theta is the new k-th distance.  For
//     k <= 256 the list lives in registers (8 keys per lane at most) and the
//     sort/merge runs on warp shuffles; above 256 both live in shared memory.
//     This replaces the per-thread insertion into an 8 KB local-memory array
//     (knnjoin.cu:774, 813-845).
// Bounds are widened by a rounding slack (bound_tol) so that FP32 rounding
// never prunes a point that the FP32 distances would rank in the top k.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "warp_select.cuh"

namespace knnsweet {

// Shared part of both top-k variants: the append buffer and the threshold.
struct TopKBase {
  uint64_t *buf;  // append buffer (shared memory)
  int nbuf, nlist, k;
  uint64_t thr;   // a candidate enters iff its key < thr
  float theta;    // distance matching thr (bound for the pruning tests)
  unsigned pushed = 0, merges = 0;  // statistics of the current query (warp-uniform)

  __device__ __forceinline__ void reset_threshold(float th0) {
    nbuf = 0;
    nlist = 0;
    theta = th0;
    // admits every d^2 <= th0^2, whatever the index
    thr = ((uint64_t)__float_as_uint(th0 * th0) << 32) | 0xffffffffull;
  }
};

// k <= 256: the sorted list of the best keys lives in registers.
template <int E>
struct RegTopK : TopKBase {
  static constexpr int L = 32 * E;
  static constexpr int kCap = L;       // candidate buffer capacity
  static constexpr int kSmemKeys = L;  // per warp
  uint64_t v[E];

  __device__ __forceinline__ int cap() const { return kCap; }

  __device__ __forceinline__ void init(uint64_t *wsm) { buf = wsm; }

  __device__ __forceinline__ void reset(float th0, int) {
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = kKeyMax;
    reset_threshold(th0);
  }

  __device__ __forceinline__ void make_room(int lane) { flush(lane); }
  // end of the query: pending candidates merged into the list
  __device__ __forceinline__ void finish(int lane) { flush(lane); }

  __device__ __forceinline__ void flush(int lane) {
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
    // both as a bitonic sequence.
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = umin64(v[j], shfl64(b[E - 1 - j], 31 - lane));
    reg_bitonic_merge<E>(v, lane);
    nlist = min(k, nlist + nbuf);
    merges++;
    nbuf = 0;
#pragma unroll
    for (int j = 0; j < E; j++)
      if (E * lane + j >= k) v[j] = kKeyMax;
    if (nlist == k) {
      const int kl = (k - 1) / E, kj = (k - 1) % E;
      uint64_t mine = kKeyMax;
#pragma unroll
      for (int j = 0; j < E; j++)
        if (j == kj) mine = v[j];
      thr = shfl64(mine, kl);
      theta = sqrtf(key_d2(thr));
    }
  }

  // Writes the k results (through the buffer for coalesced stores).
  __device__ __forceinline__ void write_out(int32_t *oi, float *od, bool squared, int32_t base, int lane) {
    __syncwarp();
#pragma unroll
    for (int j = 0; j < E; j++) buf[E * lane + j] = v[j];
    __syncwarp();
    for (int t = lane; t < k; t += 32) {
      const uint64_t key = buf[t];
      const bool none = key == kKeyMax;
      oi[t] = none ? -1 : key_idx(key) - base;
      od[t] = none ? __int_as_float(0x7f800000) : (squared ? key_d2(key) : sqrtf(key_d2(key)));
    }
    __syncwarp();
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

template <int L>
__device__ __forceinline__ void smem_bitonic_merge(uint64_t *s, int lane) {
#pragma unroll 1
  for (int stride = L >> 1; stride > 0; stride >>= 1) {
#pragma unroll
    for (int t0 = 0; t0 < (L / 2 + 31) / 32; t0++) {
      const int t = t0 * 32 + lane;
      if (t < L / 2) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const uint64_t a = s[i], b = s[j];
        if (a > b) {
          s[i] = b;
          s[j] = a;
        }
      }
    }
    __syncwarp();
  }
}

// k > 256: list and buffer both in shared memory.
template <int LL>
struct SmemTopK : TopKBase {
  static constexpr int L = LL;
  static constexpr int kCap = L;
  static constexpr int kSmemKeys = 2 * L;
  uint64_t *list;

  __device__ __forceinline__ int cap() const { return kCap; }

  __device__ __forceinline__ void init(uint64_t *wsm) {
    list = wsm;
    buf = wsm + L;
  }

  __device__ __forceinline__ void reset(float th0, int lane) {
    __syncwarp();
    for (int i = lane; i < L; i += 32) list[i] = kKeyMax;
    reset_threshold(th0);
    __syncwarp();
  }

  __device__ __forceinline__ void make_room(int lane) { flush(lane); }
  // end of the query: pending candidates merged into the list
  __device__ __forceinline__ void finish(int lane) { flush(lane); }

  __device__ __forceinline__ void flush(int lane) {
    if (nbuf == 0) return;
    __syncwarp();
    for (int i = nbuf + lane; i < L; i += 32) buf[i] = kKeyMax;
    __syncwarp();
    smem_bitonic_sort<L>(buf, lane);
    for (int i = lane; i < L; i += 32) list[i] = umin64(list[i], buf[L - 1 - i]);
    __syncwarp();
    smem_bitonic_merge<L>(list, lane);
    nlist = min(k, nlist + nbuf);
    merges++;
    nbuf = 0;
    for (int i = k + lane; i < L; i += 32) list[i] = kKeyMax;
    __syncwarp();
    if (nlist == k) {
      thr = list[k - 1];
      theta = sqrtf(key_d2(thr));
    }
  }

  __device__ __forceinline__ void write_out(int32_t *oi, float *od, bool squared, int32_t base, int lane) {
    for (int t = lane; t < k; t += 32) {
      const uint64_t key = list[t];
      const bool none = key == kKeyMax;
      oi[t] = none ? -1 : key_idx(key) - base;
      od[t] = none ? __int_as_float(0x7f800000) : (squared ? key_d2(key) : sqrtf(key_d2(key)));
    }
    __syncwarp();
  }
};

// Top-k as an unsorted candidate set in shared memory (capacity 2L).  When it
// fills, the exact k-th key is found by warp_select_kth, the set is compacted
// to the k best and the threshold drops to that key; the k results are sorted
// once, at the end of the query.
#ifndef KNN_TOPK_EARLY
#define KNN_TOPK_EARLY 160
#endif

template <int LL>
struct SelectTopK : TopKBase {
  static constexpr int L = LL;          // final sort length (pow2 >= k)
  static constexpr int kCap = 2 * LL;   // candidate capacity
  static constexpr int kSmemKeys = 2 * LL + 128;  // keys + 256-word histogram
  uint32_t *hist;

  // A compaction once k + kEarly candidates are in (capacity permitting)
  // tightens the threshold sooner.  k = 200 self-join scan: capacity only
  // 5.06 ms; kEarly 64: 5.12, 96: 4.94, 128: 4.89, 160: 4.90, 256: 4.97
  // (with the compaction before the end-of-query selection: 96: 4.86,
  // 128 to 192: 4.76-4.78).
  static constexpr int kEarly = KNN_TOPK_EARLY;
  __device__ __forceinline__ int cap() const { return k + kEarly < kCap ? k + kEarly : kCap; }

  __device__ __forceinline__ void init(uint64_t *wsm) {
    buf = wsm;
    hist = reinterpret_cast<uint32_t *>(wsm + 2 * LL);
  }

  __device__ __forceinline__ void reset(float th0, int) { reset_threshold(th0); }

  // Reduce the set to its k smallest keys (no-op with k or fewer).
  __device__ __forceinline__ void flush(int lane) {
    if (nbuf <= k) return;
    __syncwarp();
    const uint64_t kth = warp_select_kth(buf, nbuf, k, hist, lane);
    __syncwarp();
    int w = 0;
    for (int b0 = 0; b0 < nbuf; b0 += 32) {
      const int i = b0 + lane;
      const uint64_t v = i < nbuf ? buf[i] : kKeyMax;
      const bool keep = i < nbuf && v <= kth;
      const unsigned bm = __ballot_sync(kFull, keep);
      __syncwarp();
      if (keep) buf[w + __popc(bm & ((1u << lane) - 1))] = v;
      w += __popc(bm);
    }
    __syncwarp();
    nbuf = w;  // == k
    nlist = k;
    merges++;
    thr = kth;
    theta = sqrtf(key_d2(thr));
  }

  // Room for more candidates while the query runs: keep every key whose
  // squared distance is at most the k-th smallest one -- at least k keys,
  // ties included -- found by a 32-bit selection on the keys' distance words
  // (on data with many equal distances the 64-bit selection spends most of
  // its passes on the index bits of the ties).  The exact k-th key is only
  // needed at the end (flush).  Falls back to it when ties fill the buffer.
  __device__ __forceinline__ void make_room(int lane) {
    if (nbuf <= k) return;
    __syncwarp();
    const uint32_t T = warp_select_kth_u32(reinterpret_cast<const uint32_t *>(buf) + 1, 2,
                                           nbuf, k, hist, lane);
    int w = 0;
    for (int b0 = 0; b0 < nbuf; b0 += 32) {
      const int i = b0 + lane;
      const uint64_t v = i < nbuf ? buf[i] : kKeyMax;
      const bool keep = i < nbuf && (uint32_t)(v >> 32) <= T;
      const unsigned bm = __ballot_sync(kFull, keep);
      __syncwarp();
      if (keep) buf[w + __popc(bm & ((1u << lane) - 1))] = v;
      w += __popc(bm);
    }
    __syncwarp();
    nbuf = w;
    if (w > kCap - 32) {
      flush(lane);
      return;
    }
    merges++;
    thr = ((uint64_t)T << 32) | 0xffffffffull;
    theta = sqrtf(__uint_as_float(T));
  }

  // End of the query: nothing to do -- write_out sorts up to L keys as they
  // are (their first k are the answer) and selects the exact k-th key first
  // only beyond that, which saves the 64-bit selection for most queries.
  __device__ __forceinline__ void finish(int) {}

  __device__ __forceinline__ void write_out(int32_t *oi, float *od, bool squared, int32_t base, int lane) {
    // up to L keys are sorted as they are (their first k are the answer);
    // beyond that a tie-inclusive compaction first (every key at or below
    // the k-th distance stays), and the exact k-th key only if ties still
    // leave more than L
    if (nbuf > LL) make_room(lane);
    if (nbuf > LL) flush(lane);
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
      for (int j = 0; j < E; j++) {
        const int t = E * lane + j;
        if (t < k) {
          const bool none = x[j] == kKeyMax;
          oi[t] = none ? -1 : key_idx(x[j]) - base;
          od[t] = none ? __int_as_float(0x7f800000)
                       : (squared ? key_d2(x[j]) : sqrtf(key_d2(x[j])));
        }
      }
    } else {
      for (int i = nbuf + lane; i < LL; i += 32) buf[i] = kKeyMax;
      __syncwarp();
      smem_bitonic_sort<LL>(buf, lane);
      for (int t = lane; t < k; t += 32) {
        const uint64_t key = buf[t];
        const bool none = key == kKeyMax;
        oi[t] = none ? -1 : key_idx(key) - base;
        od[t] = none ? __int_as_float(0x7f800000) : (squared ? key_d2(key) : sqrtf(key_d2(key)));
      }
    }
    __syncwarp();
  }
};

// Offer one key per lane (kKeyMax = nothing); warp-collective.
template <class TK>
__device__ __forceinline__ void topk_push(TK &tk, uint64_t key, int lane) {
  bool pass = key < tk.thr;
  unsigned b = __ballot_sync(kFull, pass);
  if (b == 0) return;
  int cnt = __popc(b);
  if (tk.nbuf + cnt > tk.cap()) {
    tk.make_room(lane);
    pass = key < tk.thr;
    b = __ballot_sync(kFull, pass);
    cnt = __popc(b);
  }
  if (pass) tk.buf[tk.nbuf + __popc(b & ((1u << lane) - 1))] = key;
  tk.nbuf += cnt;
  tk.pushed += cnt;
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
// tuning knobs): the scan is latency-bound, so occupancy matters; the
// register-resident top-k needs more registers per thread.
#ifndef KNN_TARGET_WARPS_SMEM_TOPK
#define KNN_TARGET_WARPS_SMEM_TOPK 32
#endif
#ifndef KNN_TARGET_WARPS_REG_TOPK
#define KNN_TARGET_WARPS_REG_TOPK 16
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

// Largest list length kept in registers (longer lists live in shared memory).
#ifndef KNN_REG_TOPK_MAX_L
#define KNN_REG_TOPK_MAX_L 32
#endif

// Top-k for lists longer than the register limit: radix-select set
// (KNN_TOPK_SELECT=1) or sorted shared-memory list with bitonic merges.
#ifndef KNN_TOPK_SELECT
#define KNN_TOPK_SELECT 1
#endif

template <int L>
using TopKFor = std::conditional_t<
    (L <= KNN_REG_TOPK_MAX_L), RegTopK<L / 32>,
    std::conditional_t<(KNN_TOPK_SELECT != 0), SelectTopK<L>, SmemTopK<L>>>;

// Rows of more than 8 floats keep 4+ float4 of the query in registers: those
// kernels get the lower occupancy target instead of spilling.
template <int DP4, int L, int WARPS>
constexpr int scan_min_blocks() {
  return (((L <= KNN_REG_TOPK_MAX_L && L > 32) || DP4 == 0 || DP4 >= 4)
              ? KNN_TARGET_WARPS_REG_TOPK
              : KNN_TARGET_WARPS_SMEM_TOPK) /
         WARPS;
}

template <int DP4, bool IDXROW, int L, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (scan_min_blocks<DP4, L, WARPS>()))
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
  unsigned evals = 0, visited = 0, pruned = 0;
  // small rows: load the member row together with its band distance
  constexpr bool kEagerRow = KNN_EAGER_ROWS && (DP4 > 0 && DP4 <= 2);
  // statistics: per-lane 32-bit counts folded once per query into per-block
  // shared counters, added to the global ones at exit
  __shared__ unsigned long long blk_ctr[5];
  if (threadIdx.x < 5) blk_ctr[threadIdx.x] = 0;
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
    }
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
    QueryRow<DP4, IDXROW> qr;
    qr.load(a.qrows, q, dp4, qslot);
    tk.reset(a.theta0[qc], lane);

    // one band step: lane's member p of the cluster at `start`, kept when
    // its distance to the representative lies in [lo_v, hi_v]
    auto step = [&](int start, int p, bool valid, float lo_v, float hi_v) -> float {
      const int64_t gp = (int64_t)start + p;
      float dsv = 0.0f, v = 0.0f;
      int32_t idx = 0;
      bool inb;
      if constexpr (kEagerRow) {
        // small rows: issue the row load together with the band distance
        float4 row[DP4];
        if (valid) {
#pragma unroll
          for (int c = 0; c < DP4; c++) row[c] = a.srows[gp * DP4 + c];
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
          for (int c = 0; c < DP4; c++) row[c] = a.srows[gp * DP4 + c];
          v = qr.dist2_member(row, &idx);
        }
      } else {
        dsv = valid ? a.sdist[gp] : 0.0f;
        inb = valid && dsv >= lo_v && dsv <= hi_v;
        if (inb) v = qr.dist2(a.srows + gp * dp4, dp4);
      }
      uint64_t key = kKeyMax;
      if (inb) {
        evals++;
        if (v <= key_d2(tk.thr)) {
          if (!IDXROW) idx = a.sidx[gp];
          key = make_key(v, idx);
        }
      }
      topk_push(tk, key, lane);
      return dsv;
    };

    const int nr = a.rlen[qc];
    const int32_t *rl = a.rlist + (a.rl_base ? a.rl_base[qc] : (int64_t)qc * a.Rs);
    for (int base = 0; base < nr; base += 32) {
      const int j = base + lane;
      int rs = 0;
      float D = 0.0f;
      bool alive = false;
      if (j < nr) {
        rs = rl[j];
        D = sqrtf(qr.dist2(a.sreps + (int64_t)rs * dp4, dp4));
        const float th = tk.theta;
        const float slack = tol * (2.0f * D + 2.0f * th);
        alive = !(D - a.cmax[rs] > th + slack) && !(D + th + slack < a.cmin[rs]);
        if (!alive) pruned++;
      }
      // visit this chunk's surviving clusters: in list order (by rep-rep
      // distance) or, with KNN_ORDER_BY_D, nearest d(q, Rs) first
      unsigned amask = __ballot_sync(kFull, alive);
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
        const int c = __shfl_sync(kFull, rs, src);
        float th = tk.theta;
        float slack = tol * (2.0f * Dc + 2.0f * th);
        if (Dc - a.cmax[c] > th + slack || Dc + th + slack < a.cmin[c]) {
          if (lane == 0) pruned++;
          continue;
        }
        if (lane == 0) visited++;
        const int start = a.soff[c];
        const int n_c = a.soff[c + 1] - start;
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
        const int lo = lo_edge <= a.cmin[c] ? 0 : warp_lower_bound(a.sdist + start, n_c, lo_edge, lane);
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
    tk.finish(lane);
    tk.write_out(a.out_idx + q * a.k, a.out_dist + q * a.k, a.squared,
                 a.qc_ref_base ? (int32_t)a.qc_ref_base[qc] : 0, lane);
    if (a.counters) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        evals += __shfl_xor_sync(kFull, evals, o);
        visited += __shfl_xor_sync(kFull, visited, o);
        pruned += __shfl_xor_sync(kFull, pruned, o);
      }
      if (lane == 0) {
        atomicAdd(&blk_ctr[0], (unsigned long long)evals);
        atomicAdd(&blk_ctr[1], (unsigned long long)visited);
        atomicAdd(&blk_ctr[2], (unsigned long long)pruned);
        atomicAdd(&blk_ctr[3], (unsigned long long)tk.pushed);
        atomicAdd(&blk_ctr[4], (unsigned long long)tk.merges);
      }
    }
    evals = visited = pruned = 0;
    tk.pushed = tk.merges = 0;
  }
  __syncthreads();
  if (a.counters && threadIdx.x < 5) atomicAdd(a.counters + threadIdx.x, blk_ctr[threadIdx.x]);
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
  if (a.k <= 32) return launch_scan_t<DP4, IDXROW, 32, 8>(a, num_sms, s);
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
template <int DP4, bool IDXROW, int K>
__global__ void __launch_bounds__(256, 4)
    thread_scan_kernel(const ScanArgs a) {
  __shared__ unsigned long long blk_ctr[5];
  if (threadIdx.x < 5) blk_ctr[threadIdx.x] = 0;
  __syncthreads();
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nslots = a.slot_list ? (int64_t)*a.slot_count : a.m;
  unsigned evals = 0, visited = 0, pruned = 0, pushed = 0;
  if (t < nslots) {
    const int64_t slot = a.slot_list ? (int64_t)a.slot_list[t] : t;
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
    const float tol = bound_tol(a.d);
    QueryRow<DP4, IDXROW> qr;
    qr.load(a.qrows, q, DP4, nullptr);
    ThreadTopK<K> tk;
    tk.reset();
    float theta = a.theta0[qc];
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
        pruned++;
        continue;
      }
      visited++;
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
        if (key < thr0 && key < tk.key[K - 1]) {
          tk.insert(key);
          pushed++;
          if (tk.key[K - 1] != kKeyMax) {
            theta = sqrtf(key_d2(tk.key[K - 1]));
            slack = tol * (2.0f * D + 2.0f * theta);
          }
        }
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
  }
  if (a.counters) {
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
    if (threadIdx.x < 5) atomicAdd(a.counters + threadIdx.x, blk_ctr[threadIdx.x]);
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

#ifndef KNN_THREAD_SCAN_MAX_K
#define KNN_THREAD_SCAN_MAX_K 32
#endif

int launch_scan(const ScanArgs &a, int num_sms, cudaStream_t s) {
  if (a.m == 0) return KNN_OK;
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
