// bounds.cuh -- per query cluster k-th bound and reference-cluster filter,
// as a block-level device function shared by the single join
// (bounds_filter_kernel) and the batched join (batched_bounds_kernel).
#pragma once

#include "common.cuh"
#include "warp_select.cuh"

namespace knnsweet {

// ---------------------------------------------------------------------------
// Per query cluster (one block each):
//  1. theta0 = k-th smallest over all reference points s of
//     rq + d(Rq, Rs(s)) + d(s, Rs(s)), the bound RepsUpperBound computes
//     (knnjoin.cu:459-504), found exactly by bisection on the value's bit
//     pattern with a count of values <= T (binary search per cluster over its
//     first min(k, size) members).  The reference keeps the K smallest in a
//     list and replaces every entry equal to the maximum at once (486-489,
//     defect B2), which undercounts ties; the count here is exact.  Widened
//     by the rounding slack.
//  2. The reference clusters Rs that can hold a point within theta0 of some
//     query of the cluster: d(Rq,Rs) - rq - radius(Rs) <= theta0
//     (FilterReps, knnjoin.cu:506-525), sorted by d(Rq,Rs), then Rs
//     (the host std::sort of knnjoin.cu:1080-1091); only the survivors
//     enter the sort.
// ---------------------------------------------------------------------------
// One query cluster's bound and candidate list, by one block.  The reference
// clusters are the Rs_loc consecutive clusters whose offsets start at soff
// (soff[0] .. soff[Rs_loc]; their points are sdist[soff[j] ..]); dq[j] is the
// distance from this query cluster's representative to theirs.  Writes
// theta0, the surviving clusters (as id_base + j, nearest first) and their
// count.  skey: rs_pow2 >= Rs_loc keys of dynamic shared memory.
static __device__ __forceinline__ void bounds_filter_block(const float *dq, int Rs_loc, const int32_t *__restrict__ soff,
                                    const float *__restrict__ sdist,
                                    const float *__restrict__ scmax, float rq, int k, int d,
                                    int rs_pow2, int32_t id_base, uint64_t *skey,
                                    float *theta0_out, int32_t *rlist_out,
                                    int32_t *rlen_out, float2 *chunk_out = nullptr) {
  __shared__ int red_i[32];
  __shared__ unsigned red_u[32], red_l[32];
  __shared__ int kept_s;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nth >> 5;
  const float tol = bound_tol(d);
  const int64_t n = soff[Rs_loc] - soff[0];
  const int kk = (int)(k < n ? k : n);
  if (kk == 0) {
    if (tid == 0) {
      *theta0_out = 0.0f;
      *rlen_out = 0;
    }
    return;
  }

  // upper end of the bisection: the largest value any cluster contributes,
  // or better, the kk-th value of any single cluster holding kk members
  // (that cluster alone has kk values at or below it).  Each cluster's
  // smallest value is kept in shared memory (the sort keys' space, reused
  // below): a cluster whose smallest value exceeds T adds nothing to the
  // count at T and skips its search.
  float *lo_v = reinterpret_cast<float *>(skey);
  unsigned hi_local = 0, u_local = 0xffffffffu, l_local = 0xffffffffu;
  for (int j = tid; j < Rs_loc; j += nth) {
    int a = soff[j], sz = min(soff[j + 1] - a, kk);
    float first = __int_as_float(0x7f800000);
    if (sz > 0) {
      const float base = __fadd_rn(rq, dq[j]);
      float v = __fadd_rn(base, sdist[a + sz - 1]);
      hi_local = max(hi_local, __float_as_uint(v));
      if (sz == kk) u_local = min(u_local, __float_as_uint(v));
      first = __fadd_rn(base, sdist[a]);
      l_local = min(l_local, __float_as_uint(first));
    }
    lo_v[j] = first;
  }
  for (int o = 16; o > 0; o >>= 1) {
    hi_local = max(hi_local, __shfl_xor_sync(kFull, hi_local, o));
    u_local = min(u_local, __shfl_xor_sync(kFull, u_local, o));
    l_local = min(l_local, __shfl_xor_sync(kFull, l_local, o));
  }
  if (lane == 0) {
    red_u[warp] = hi_local;
    red_i[warp] = (int)u_local;
    red_l[warp] = l_local;
  }
  __syncthreads();
  unsigned hi = 0, u = 0xffffffffu, lo = 0xffffffffu;
  for (int w = 0; w < nwarp; w++) {
    hi = max(hi, red_u[w]);
    u = min(u, (unsigned)red_i[w]);
    lo = min(lo, red_l[w]);
  }
  if (u < hi) hi = u;
  __syncthreads();
  // smallest bit pattern T with count(values <= T) >= kk; count(hi) >= kk.
  // lo: the smallest value of all (nothing lies below it), lo <= hi
  // invariant: answer in [lo, hi]
  while (lo < hi) {
    unsigned mid = lo + ((hi - lo) >> 1);
    float T = __uint_as_float(mid);
    int cnt = 0;
    for (int j = tid; j < Rs_loc; j += nth) {
      if (lo_v[j] > T) continue;  // empty cluster (+inf) or nothing <= T
      int a = soff[j], sz = min(soff[j + 1] - a, kk);
      float base = __fadd_rn(rq, dq[j]);
      int l = 0, h = sz;  // first t with base + sdist[a+t] > T
      while (l < h) {
        int md = (l + h) >> 1;
        if (__fadd_rn(base, sdist[a + md]) <= T) l = md + 1;
        else h = md;
      }
      cnt += l;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kFull, cnt, o);
    if (lane == 0) red_i[warp] = cnt;
    __syncthreads();
    int total = 0;
    for (int w = 0; w < nwarp; w++) total += red_i[w];
    __syncthreads();
    if (total >= kk) hi = mid;
    else lo = mid + 1;
  }
  const float kth = __uint_as_float(hi);
  const float th = __fmaf_rn(kth, 4.0f * tol, kth) + 1.17549435e-38f;
  if (tid == 0) {
    *theta0_out = th;
    kept_s = 0;
  }
  __syncthreads();

  // filter: the survivors are compacted into skey (in any order; the keys
  // are distinct), then only those are sorted by (d(Rq,Rs), Rs)
  for (int j = tid; j < Rs_loc; j += nth) {
    if (soff[j + 1] > soff[j]) {
      float dd = dq[j], rr = scmax[j];
      float lb = dd - rq - rr;
      if (!(lb > th + tol * (dd + rq + rr + th)))
        skey[atomicAdd(&kept_s, 1)] = ((uint64_t)__float_as_uint(dd) << 32) | (uint32_t)j;
    }
  }
  __syncthreads();
  int p2 = 1;  // <= rs_pow2: a power of two >= Rs_loc >= kept
  while (p2 < kept_s) p2 <<= 1;
  for (int j = kept_s + tid; j < p2; j += nth) skey[j] = kKeyMax;
  __syncthreads();
  for (int size = 2; size <= p2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = tid; t < (p2 >> 1); t += nth) {
        int i = 2 * t - (t & (stride - 1));
        int j = i + stride;
        bool up = (i & size) == 0;
        uint64_t a = skey[i], b = skey[j];
        if ((a > b) == up) {
          skey[i] = b;
          skey[j] = a;
        }
      }
      __syncthreads();
    }
  }
  const int kept = kept_s;
  for (int j = tid; j < kept; j += nth)
    rlist_out[j] = id_base + (int32_t)(skey[j] & 0xffffffffu);
  if (tid == 0) *rlen_out = kept;
  if (chunk_out && warp == 0) {
    // per chunk of 32 list entries: the first entry's d(Rq, Rs) (the list
    // is ascending in it) and the largest radius from that entry to the end,
    // by suffix maxima over the chunks, 32 chunks per round from the back
    const int nch = (kept + 31) >> 5;
    float carry = 0.0f;
    for (int c0 = (nch - 1) & ~31; c0 >= 0; c0 -= 32) {
      const int c = c0 + lane;
      float m = 0.0f, first = 0.0f;
      if (c < nch) {
        const int e1 = min(32 * c + 32, kept);
        for (int e = 32 * c; e < e1; e++)
          m = fmaxf(m, scmax[(int32_t)(skey[e] & 0xffffffffu)]);
        first = __uint_as_float((uint32_t)(skey[32 * c] >> 32));
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_down_sync(kFull, m, o);
        if (lane + o < 32) m = fmaxf(m, t);
      }
      m = fmaxf(m, carry);
      carry = __shfl_sync(kFull, m, 0);
      if (c < nch) chunk_out[c] = make_float2(first, m);
    }
  }
}

// The same bound and candidate list by one warp, for query clusters with few
// reference clusters (the batched form: one cloud's representatives, a few
// hundred at most).  Identical arithmetic -- the bisection counts, the filter
// test and the sort keys are the block version's -- with shuffle reductions
// instead of block barriers and a ballot compaction of the survivors (the
// sort makes their order the same).  skey: rs_pow2 >= Rs_loc keys of this
// warp's shared memory.
static __device__ __forceinline__ void bounds_filter_warp(
    const float *dq, int Rs_loc, const int32_t *__restrict__ soff,
    const float *__restrict__ sdist, const float *__restrict__ scmax, float rq, int k, int d,
    int32_t id_base, uint64_t *skey, float *theta0_out, int32_t *rlist_out,
    int32_t *rlen_out, int lane) {
  const float tol = bound_tol(d);
  const int64_t n = soff[Rs_loc] - soff[0];
  const int kk = (int)(k < n ? k : n);
  if (kk == 0) {
    if (lane == 0) {
      *theta0_out = 0.0f;
      *rlen_out = 0;
    }
    return;
  }
  float *lo_v = reinterpret_cast<float *>(skey);
  unsigned hi = 0, u = 0xffffffffu, lo = 0xffffffffu;
  for (int j = lane; j < Rs_loc; j += 32) {
    const int a = soff[j], sz = min(soff[j + 1] - a, kk);
    float first = __int_as_float(0x7f800000);
    if (sz > 0) {
      const float base = __fadd_rn(rq, dq[j]);
      const float v = __fadd_rn(base, sdist[a + sz - 1]);
      hi = max(hi, __float_as_uint(v));
      if (sz == kk) u = min(u, __float_as_uint(v));
      first = __fadd_rn(base, sdist[a]);
      lo = min(lo, __float_as_uint(first));
    }
    lo_v[j] = first;
  }
  hi = __reduce_max_sync(kFull, hi);
  u = __reduce_min_sync(kFull, u);
  lo = __reduce_min_sync(kFull, lo);
  if (u < hi) hi = u;
  __syncwarp();
  // smallest bit pattern T with count(values <= T) >= kk, in [lo, hi]
  while (lo < hi) {
    const unsigned mid = lo + ((hi - lo) >> 1);
    const float T = __uint_as_float(mid);
    int cnt = 0;
    for (int j = lane; j < Rs_loc; j += 32) {
      if (lo_v[j] > T) continue;
      const int a = soff[j], sz = min(soff[j + 1] - a, kk);
      const float base = __fadd_rn(rq, dq[j]);
      int l = 0, h = sz;
      while (l < h) {
        const int md = (l + h) >> 1;
        if (__fadd_rn(base, sdist[a + md]) <= T) l = md + 1;
        else h = md;
      }
      cnt += l;
    }
    if ((int)__reduce_add_sync(kFull, (unsigned)cnt) >= kk) hi = mid;
    else lo = mid + 1;
  }
  const float kth = __uint_as_float(hi);
  const float th = __fmaf_rn(kth, 4.0f * tol, kth) + 1.17549435e-38f;
  __syncwarp();
  // survivors compacted in cluster order, then sorted by (d(Rq,Rs), Rs)
  int kept = 0;
  for (int j0 = 0; j0 < Rs_loc; j0 += 32) {
    const int j = j0 + lane;
    bool keep = false;
    uint64_t key = 0;
    if (j < Rs_loc && soff[j + 1] > soff[j]) {
      const float dd = dq[j], rr = scmax[j];
      const float lb = dd - rq - rr;
      keep = !(lb > th + tol * (dd + rq + rr + th));
      key = ((uint64_t)__float_as_uint(dd) << 32) | (uint32_t)j;
    }
    const unsigned bm = __ballot_sync(kFull, keep);
    if (keep) skey[kept + __popc(bm & ((1u << lane) - 1u))] = key;
    kept += __popc(bm);
  }
  int p2 = 1;
  while (p2 < kept) p2 <<= 1;
  for (int j = kept + lane; j < p2; j += 32) skey[j] = kKeyMax;
  __syncwarp();
  smem_bitonic_sort_rt(skey, p2, lane);
  for (int j = lane; j < kept; j += 32) rlist_out[j] = id_base + (int32_t)(skey[j] & 0xffffffffu);
  if (lane == 0) {
    *theta0_out = th;
    *rlen_out = kept;
  }
}

}  // namespace knnsweet
