// scan.cu -- the per-query pruned scan (replaces KNNQuery_base,
// src/knnjoin.cu:762-858, and the small-M KNNQuery + final merge,
// src/knnjoin.cu:859-979).
//
// One warp per query, persistent blocks pulling query slots from an atomic
// counter in query-cluster order (the reference's reorder_members,
// knnjoin.cu:114-124, 768), so neighbouring warps walk the same candidate
// list.  For every surviving reference cluster Rs of the query's cluster
// (nearest representative first):
//   - 32 clusters at a time, each lane computes D = d(q, Rs) and drops the
//     cluster if  D - radius(Rs) > theta  or  D + theta < min member
//     distance: no member can be within theta (the reference's first-member
//     `break`, knnjoin.cu:797).
//   - Members are stored contiguously, ascending by d(s, Rs).  The members
//     that can be within theta of q satisfy |D - d(s,Rs)| <= theta
//     (knnjoin.cu:796-801), a contiguous band: its lower end is found by a
//     warp-wide 32-ary search, and the warp walks the band 32 members per
//     step with coalesced float4 row loads, stopping as soon as a whole step
//     lies above D + theta.
//   - Exact FP32 distances of band members go through the warp top-k:
//     candidates whose (d^2, index) key beats the current k-th key are
//     appended to a shared-memory buffer; a full buffer is bitonic-sorted and
//     merged into the sorted list of the k best, and theta drops to the new
//     k-th distance.  This replaces the per-thread insertion sort into an
//     8 KB local-memory array (knnjoin.cu:774, 813-845).
// Bounds are widened by a rounding slack (bound_tol) so that FP32 rounding
// never prunes a point that the FP32 distances would rank in the top k.
#include "common.cuh"
#include "kernels.cuh"

namespace knnsweet {

// Bitonic sort of L keys in shared memory, ascending, by one warp.
template <int L>
__device__ __forceinline__ void warp_bitonic_sort(uint64_t *s, int lane) {
#pragma unroll 1
  for (int size = 2; size <= L; size <<= 1) {
#pragma unroll 1
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
      for (int t0 = 0; t0 < (L / 2 + 31) / 32; t0++) {
        int t = t0 * 32 + lane;
        if (t < L / 2) {
          int i = 2 * t - (t & (stride - 1));
          int j = i + stride;
          bool up = (i & size) == 0;
          uint64_t a = s[i], b = s[j];
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

// Sorts a bitonic sequence of L keys ascending (half-cleaner cascade).
template <int L>
__device__ __forceinline__ void warp_bitonic_merge(uint64_t *s, int lane) {
#pragma unroll 1
  for (int stride = L >> 1; stride > 0; stride >>= 1) {
#pragma unroll
    for (int t0 = 0; t0 < (L / 2 + 31) / 32; t0++) {
      int t = t0 * 32 + lane;
      if (t < L / 2) {
        int i = 2 * t - (t & (stride - 1));
        int j = i + stride;
        uint64_t a = s[i], b = s[j];
        if (a > b) {
          s[i] = b;
          s[j] = a;
        }
      }
    }
    __syncwarp();
  }
}

// Warp-wide top-k state: `list` holds the nlist best keys (ascending, the
// rest kKeyMax), `buf` the nbuf not yet merged candidates, `thr` the key a
// candidate must beat and `theta` the matching distance.
template <int L>
struct WarpTopK {
  uint64_t *list;
  uint64_t *buf;
  int nlist, nbuf, k;
  uint64_t thr, thr0;
  float theta, theta0;

  __device__ __forceinline__ void reset(float th0, int lane) {
    for (int i = lane; i < L; i += 32) list[i] = kKeyMax;
    nlist = 0;
    nbuf = 0;
    theta0 = th0;
    theta = th0;
    // admits every d^2 <= th0^2, whatever the index
    thr0 = ((uint64_t)__float_as_uint(th0 * th0) << 32) | 0xffffffffull;
    thr = thr0;
    __syncwarp();
  }

  __device__ __forceinline__ void flush(int lane) {
    if (nbuf == 0) return;
    __syncwarp();
    for (int i = nbuf + lane; i < L; i += 32) buf[i] = kKeyMax;
    __syncwarp();
    warp_bitonic_sort<L>(buf, lane);
    for (int i = lane; i < L; i += 32) {
      uint64_t a = list[i], b = buf[L - 1 - i];
      list[i] = a < b ? a : b;
    }
    __syncwarp();
    warp_bitonic_merge<L>(list, lane);
    nlist = min(k, nlist + nbuf);
    nbuf = 0;
    for (int i = k + lane; i < L; i += 32) list[i] = kKeyMax;
    __syncwarp();
    if (nlist == k) {
      thr = list[k - 1];
      theta = sqrtf(key_d2(thr));
    }
  }

  // Offer one key per lane (kKeyMax = nothing).
  __device__ __forceinline__ void push(uint64_t key, int lane) {
    bool pass = key < thr;
    unsigned b = __ballot_sync(kFull, pass);
    if (b == 0) return;
    int cnt = __popc(b);
    if (nbuf + cnt > L) {
      flush(lane);
      pass = key < thr;
      b = __ballot_sync(kFull, pass);
      cnt = __popc(b);
    }
    if (pass) buf[nbuf + __popc(b & ((1u << lane) - 1))] = key;
    nbuf += cnt;
  }
};

template <int DP4>
struct QueryRow {
  float4 v[DP4];
  __device__ __forceinline__ void load(const float4 *__restrict__ rows,
                                       int64_t q, int, float4 *) {
#pragma unroll
    for (int c = 0; c < DP4; c++) v[c] = rows[q * DP4 + c];
  }
  __device__ __forceinline__ float dist2(const float4 *__restrict__ r, int) const {
    return dist2_rows<DP4>(v, r);
  }
};

// Runtime width: the query row lives in the warp's shared-memory slot.
template <>
struct QueryRow<0> {
  const float4 *v;
  __device__ __forceinline__ void load(const float4 *__restrict__ rows,
                                       int64_t q, int dp4, float4 *slot) {
    int lane = threadIdx.x & 31;
    __syncwarp();
    for (int c = lane; c < dp4; c += 32) slot[c] = rows[q * dp4 + c];
    __syncwarp();
    v = slot;
  }
  __device__ __forceinline__ float dist2(const float4 *__restrict__ r, int dp4) const {
    return dist2_rows_rt(v, r, dp4);
  }
};

template <int DP4, int L, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    scan_kernel(const ScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int dp4 = DP4 > 0 ? DP4 : a.dp4;
  uint64_t *wsm = reinterpret_cast<uint64_t *>(smem_raw) + (size_t)w * 2 * L;
  float4 *qslot = reinterpret_cast<float4 *>(
                      reinterpret_cast<uint64_t *>(smem_raw) + (size_t)WARPS * 2 * L) +
                  (size_t)w * (DP4 > 0 ? 0 : a.dp4);
  WarpTopK<L> tk;
  tk.list = wsm;
  tk.buf = wsm + L;
  tk.k = a.k;
  const float tol = bound_tol(a.d);
  unsigned long long evals = 0, visited = 0, pruned = 0;

  for (;;) {
    long long slot = 0;
    if (lane == 0) slot = (long long)atomicAdd(a.work_counter, 1ull);
    slot = __shfl_sync(kFull, slot, 0);
    if (slot >= a.m) break;
    const int64_t q = a.qorder[slot];
    const int qc = a.slot_cl[slot];
    QueryRow<DP4> qr;
    qr.load(a.qrows, q, dp4, qslot);
    tk.reset(a.theta0[qc], lane);

    const int nr = a.rlen[qc];
    const int32_t *rl = a.rlist + (int64_t)qc * a.Rs;
    for (int base = 0; base < nr; base += 32) {
      const int j = base + lane;
      int rs = 0;
      float D = 0.0f;
      bool alive = false;
      if (j < nr) {
        rs = rl[j];
        D = sqrtf(qr.dist2(a.sreps + (int64_t)rs * dp4, dp4));
        float th = tk.theta;
        float slack = tol * (2.0f * D + 2.0f * th);
        alive = !(D - a.cmax[rs] > th + slack) && !(D + th + slack < a.cmin[rs]);
        if (!alive) pruned++;
      }
      unsigned mask = __ballot_sync(kFull, alive);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const int c = __shfl_sync(kFull, rs, src);
        const float Dc = __shfl_sync(kFull, D, src);
        float th = tk.theta;
        float slack = tol * (2.0f * Dc + 2.0f * th);
        if (Dc - a.cmax[c] > th + slack || Dc + th + slack < a.cmin[c]) {
          if (lane == 0) pruned++;
          continue;
        }
        if (lane == 0) visited++;
        const int start = a.soff[c], end = a.soff[c + 1];
        const int lo = warp_lower_bound(a.sdist + start, end - start,
                                        Dc - th - slack, lane);
        for (int p0 = start + lo; p0 < end; p0 += 32) {
          const int p = p0 + lane;
          th = tk.theta;
          slack = tol * (2.0f * Dc + 2.0f * th);
          const float up = Dc + th + slack, dn = Dc - th - slack;
          const bool valid = p < end;
          const float dsv = valid ? a.sdist[p] : 0.0f;
          const bool inb = valid && dsv <= up && dsv >= dn;
          uint64_t key = kKeyMax;
          if (inb) {
            const float v = qr.dist2(a.srows + (int64_t)p * dp4, dp4);
            evals++;
            if (v <= key_d2(tk.thr)) key = make_key(v, a.sidx[p]);
          }
          tk.push(key, lane);
          const bool past = !valid || dsv > up;
          if (__shfl_sync(kFull, past, 31)) break;
        }
      }
    }
    tk.flush(lane);
    int32_t *oi = a.out_idx + q * a.k;
    float *od = a.out_dist + q * a.k;
    for (int t = lane; t < a.k; t += 32) {
      uint64_t key = tk.list[t];
      bool none = key == kKeyMax;
      oi[t] = none ? -1 : key_idx(key);
      od[t] = none ? __int_as_float(0x7f800000) : sqrtf(key_d2(key));
    }
    __syncwarp();
  }
  // one atomic per warp for each statistic
  for (int o = 16; o > 0; o >>= 1) {
    evals += __shfl_xor_sync(kFull, evals, o);
    visited += __shfl_xor_sync(kFull, visited, o);
    pruned += __shfl_xor_sync(kFull, pruned, o);
  }
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, evals);
    atomicAdd(a.counters + 1, visited);
    atomicAdd(a.counters + 2, pruned);
  }
}

template <int DP4, int L, int WARPS>
static int launch_scan_t(const ScanArgs &a, int num_sms, cudaStream_t s) {
  size_t smem = (size_t)WARPS * 2 * L * sizeof(uint64_t) +
                (DP4 > 0 ? 0 : (size_t)WARPS * a.dp4 * sizeof(float4));
  auto kern = scan_kernel<DP4, L, WARPS>;
  if (smem > 48 * 1024)
    KNN_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  int per_sm = 0;
  KNN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem));
  if (per_sm < 1) per_sm = 1;
  int64_t want = (a.m + WARPS - 1) / WARPS;
  int64_t grid = (int64_t)num_sms * per_sm;
  if (grid > want) grid = want;
  if (grid < 1) grid = 1;
  kern<<<(int)grid, WARPS * 32, smem, s>>>(a);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

template <int DP4>
static int launch_scan_l(const ScanArgs &a, int num_sms, cudaStream_t s) {
  if (a.k <= 32) return launch_scan_t<DP4, 32, 8>(a, num_sms, s);
  if (a.k <= 64) return launch_scan_t<DP4, 64, 8>(a, num_sms, s);
  if (a.k <= 128) return launch_scan_t<DP4, 128, 8>(a, num_sms, s);
  if (a.k <= 256) return launch_scan_t<DP4, 256, 8>(a, num_sms, s);
  if (a.k <= 512) return launch_scan_t<DP4, 512, 4>(a, num_sms, s);
  return launch_scan_t<DP4, 1024, 4>(a, num_sms, s);
}

int launch_scan(const ScanArgs &a, int num_sms, cudaStream_t s) {
  if (a.m == 0) return KNN_OK;
  switch (a.dp4_tmpl) {
    case 1: return launch_scan_l<1>(a, num_sms, s);
    case 2: return launch_scan_l<2>(a, num_sms, s);
    case 4: return launch_scan_l<4>(a, num_sms, s);
    case 8: return launch_scan_l<8>(a, num_sms, s);
    default: return launch_scan_l<0>(a, num_sms, s);
  }
}

}  // namespace knnsweet
