// warp_select.cuh -- warp-level helpers on 64-bit (distance, index) keys
// shared by the pruned scan and the tensor-core tile search: 64-bit
// shuffles, the exact k-th key by radix selection, bitonic networks in
// registers and a runtime-length bitonic sort in shared memory.
#pragma once

#include "common.cuh"

// Compactions that only need a pruning threshold (the scan's mid-query
// candidate set, the tile search's bound buffer) select an upper bound of the
// k-th value from one linear-bin histogram pass (1) or the exact k-th by
// radix selection (0).
#ifndef KNN_LINEAR_SELECT
#define KNN_LINEAR_SELECT 1
#endif
// Final sorts of 129 to 256 candidate keys: binned counting sort (1) or the
// shared-memory bitonic network (0).
#ifndef KNN_BIN_SORT
#define KNN_BIN_SORT 1
#endif

namespace knnsweet {

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
  uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
  uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ __forceinline__ uint64_t umax64(uint64_t a, uint64_t b) { return a < b ? b : a; }

// k-th smallest (1-based rank k, 1 <= k <= n) of the distinct keys s[0..n),
// by one warp: radix selection with 8-bit digits, starting at the highest bit
// in which the keys differ; `hist` is a 256-word shared-memory histogram.
// (Inlined: an out-of-line call spilled the caller's registers around it.)
__device__ __forceinline__ uint64_t warp_select_kth(const uint64_t *s, int n, int k,
                                                 uint32_t *hist, int lane) {
  uint64_t mn = kKeyMax, mx = 0;
  for (int i = lane; i < n; i += 32) {
    const uint64_t v = s[i];
    mn = umin64(mn, v);
    mx = umax64(mx, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = umin64(mn, shfl_xor64(mn, o));
    mx = umax64(mx, shfl_xor64(mx, o));
  }
  if (mn == mx) return mn;
  const int hb = 63 - __clzll((long long)(mn ^ mx));  // highest differing bit
  uint64_t known = hb == 63 ? 0ull : (~0ull << (hb + 1));
  uint64_t prefix = mn & known;
  uint32_t need = (uint32_t)k;
  int top = hb + 1;  // bits [0, top) still unknown
  for (;;) {
    const int shift = top > 8 ? top - 8 : 0;
    const uint32_t dmask = (1u << (top - shift)) - 1u;
    __syncwarp();
#pragma unroll
    for (int b = 0; b < 8; b++) hist[b * 32 + lane] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      const uint64_t v = s[i];
      if ((v & known) == prefix) atomicAdd(&hist[(uint32_t)(v >> shift) & dmask], 1u);
    }
    __syncwarp();
    // bin holding the need-th key: scan the bins 32 at a time
    uint32_t base = 0, before = 0, cnt_b = 0;
    int bin = -1;
#pragma unroll 1
    for (int j = 0; j < 8 && bin < 0; j++) {
      const uint32_t h = hist[j * 32 + lane];
      uint32_t incl = h;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const uint32_t total = __shfl_sync(kFull, incl, 31);
      if (base + total >= need) {
        const int wl = __ffs(__ballot_sync(kFull, base + incl >= need)) - 1;
        bin = j * 32 + wl;
        before = base + __shfl_sync(kFull, incl - h, wl);
        cnt_b = __shfl_sync(kFull, h, wl);
      }
      base += total;
    }
    need -= before;
    prefix |= (uint64_t)bin << shift;
    known |= (uint64_t)dmask << shift;
    if (shift == 0) return prefix;
    if (cnt_b == 1) {  // the only key with this prefix
      uint64_t found = 0;
      bool f = false;
      for (int i = lane; i < n; i += 32) {
        const uint64_t v = s[i];
        if ((v & known) == prefix) {
          found = v;
          f = true;
        }
      }
      return shfl64(found, __ffs(__ballot_sync(kFull, f)) - 1);
    }
    top = shift;
  }
}

// k-th smallest (1-based, 1 <= k <= n) of the 32-bit values s[i * stride],
// i < n, which may repeat: the value v with #{s < v} < k <= #{s <= v}.  One
// warp, 8-bit digit passes over s (global or shared memory) restricted to the
// bits that differ between the values -- an OR / AND pass finds them; on
// small integers stored as floats (squared distances of integer points) the
// low mantissa bits are all zero and two passes replace four.  `hist` is a
// 256-word shared-memory histogram.  Non-negative floats order like their
// bit patterns, so this also selects among non-negative floats.
__device__ __forceinline__ uint32_t warp_select_kth_u32(const uint32_t *s, int stride, int n,
                                                        int k, uint32_t *hist, int lane) {
  uint32_t vor = 0u, vand = 0xffffffffu;
  for (int i = lane; i < n; i += 32) {
    const uint32_t v = s[(size_t)i * stride];
    vor |= v;
    vand &= v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vor |= __shfl_xor_sync(kFull, vor, o);
    vand &= __shfl_xor_sync(kFull, vand, o);
  }
  const uint32_t diff = vor ^ vand;  // bits in which some values differ
  if (diff == 0u) return vand;       // all equal
  const int hb = 31 - __clz(diff), lb = __ffs(diff) - 1;
  // bits above hb and below lb are the same in every value
  uint32_t known = hb == 31 ? 0u : (0xffffffffu << (hb + 1));
  uint32_t prefix = vand & known, need = (uint32_t)k;
#pragma unroll 1
  for (int top = hb + 1; top > lb;) {
    const int shift = top - 8 > lb ? top - 8 : lb;
    const uint32_t dmask = (1u << (top - shift)) - 1u;
    __syncwarp();
#pragma unroll
    for (int b = 0; b < 8; b++) hist[b * 32 + lane] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      const uint32_t v = s[(size_t)i * stride];
      if ((v & known) == prefix) atomicAdd(&hist[(v >> shift) & dmask], 1u);
    }
    __syncwarp();
    uint32_t base = 0, before = 0;
    int bin = -1;
#pragma unroll 1
    for (int j = 0; j < 8 && bin < 0; j++) {
      const uint32_t h = hist[j * 32 + lane];
      uint32_t incl = h;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const uint32_t total = __shfl_sync(kFull, incl, 31);
      if (base + total >= need) {
        const int wl = __ffs(__ballot_sync(kFull, base + incl >= need)) - 1;
        bin = j * 32 + wl;
        before = base + __shfl_sync(kFull, incl - h, wl);
      }
      base += total;
    }
    need -= before;
    prefix |= (uint32_t)bin << shift;
    known |= dmask << shift;
    top = shift;
  }
  __syncwarp();
  return prefix | (vand & ((1u << lb) - 1u));  // the common low bits
}

// An upper bound of the k-th smallest (1-based, 1 <= k <= n) of the
// non-negative floats s[i * stride], i < n (as bit patterns), that is itself
// one of the values: the largest value of the bin holding the k-th, the bins
// splitting [min, max] into 128 equal parts.  bin(v) is non-decreasing in v
// (subtraction, multiplication by a positive factor and truncation all are),
// so the values of the bins up to that bin are the smallest ones and the k-th
// lies among them.  One min / max pass and one histogram pass (counts and
// per-bin maxima, `hist`: 256 shared words), against two to four passes of
// the exact radix selection; for a pruning threshold an upper bound is as
// good as the k-th itself.
__device__ __forceinline__ uint32_t warp_kth_upper_u32(const uint32_t *s, int stride, int n,
                                                       int k, uint32_t *hist, int lane) {
  uint32_t mn = 0xffffffffu, mx = 0u;
  for (int i = lane; i < n; i += 32) {
    const uint32_t v = s[(size_t)i * stride];
    mn = min(mn, v);
    mx = max(mx, v);
  }
  mn = __reduce_min_sync(kFull, mn);
  mx = __reduce_max_sync(kFull, mx);
  if (mn == mx) return mx;
  const float fmn = __uint_as_float(mn);
  const float scale = fminf(128.0f / (__uint_as_float(mx) - fmn), 1e30f);
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 8; b++) hist[b * 32 + lane] = 0;
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    const uint32_t v = s[(size_t)i * stride];
    const int b = min((int)((__uint_as_float(v) - fmn) * scale), 127);
    atomicAdd(&hist[b], 1u);
    atomicMax(&hist[128 + b], v);
  }
  __syncwarp();
  uint32_t base = 0;
  int bin = 127;
#pragma unroll 1
  for (int j = 0; j < 4; j++) {
    const uint32_t h = hist[j * 32 + lane];
    uint32_t incl = h;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (base + total >= (uint32_t)k) {
      bin = j * 32 + __ffs(__ballot_sync(kFull, base + incl >= (uint32_t)k)) - 1;
      break;
    }
    base += total;
  }
  const uint32_t r = hist[128 + bin];
  __syncwarp();
  return r;
}

// Sorts the n <= 32*E distinct keys s[0..n) ascending, by one warp, in three
// passes instead of a bitonic network: the keys are counted into 128 linear
// bins of their distance words between the smallest and the largest (bin(v)
// non-decreasing in v, so bins hold consecutive runs of the sorted order), an
// exclusive scan gives every bin its first position, the keys are placed bin
// by bin into tmp (n keys of scratch), and every key then moves to its bin's
// first position plus its rank among the keys of its bin.  Returns false,
// having changed nothing, when a bin holds more than kMaxBin keys (many equal
// distances: the rank loop would cost more than the network).  `hist`: 256
// shared words.
template <int E>
__device__ __forceinline__ bool warp_bin_sort(uint64_t *s, int n, uint64_t *tmp,
                                              uint32_t *hist, int lane) {
  constexpr uint32_t kMaxBin = 48;
  uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int i = j * 32 + lane;
    if (i < n) {
      const uint32_t v = (uint32_t)(s[i] >> 32);
      mn = min(mn, v);
      mx = max(mx, v);
    }
  }
  mn = __reduce_min_sync(kFull, mn);
  mx = __reduce_max_sync(kFull, mx);
  const float fmn = __uint_as_float(mn);
  const float scale = mx > mn ? fminf(128.0f / (__uint_as_float(mx) - fmn), 1e30f) : 0.0f;
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 4; b++) hist[b * 32 + lane] = 0;
  __syncwarp();
  uint32_t tag[E];  // bin << 16 | place inside the bin
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int i = j * 32 + lane;
    tag[j] = 0;
    if (i < n) {
      const float v = __uint_as_float((uint32_t)(s[i] >> 32));
      const uint32_t b = (uint32_t)min((int)((v - fmn) * scale), 127);
      tag[j] = (b << 16) | atomicAdd(&hist[b], 1u);
    }
  }
  __syncwarp();
  uint32_t base = 0, big = 0;
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    const uint32_t h = hist[jj * 32 + lane];
    big = max(big, h);
    uint32_t incl = h;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    hist[128 + jj * 32 + lane] = base + incl - h;
    base += __shfl_sync(kFull, incl, 31);
  }
  if (__reduce_max_sync(kFull, big) > kMaxBin) return false;
  __syncwarp();
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int i = j * 32 + lane;
    if (i < n) tmp[hist[128 + (tag[j] >> 16)] + (tag[j] & 0xffffu)] = s[i];
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int i = j * 32 + lane;
    if (i < n) {
      const uint32_t b = tag[j] >> 16, st = hist[128 + b], cnt = hist[b];
      const uint64_t key = tmp[st + (tag[j] & 0xffffu)];
      uint32_t r = 0;
      for (uint32_t t = 0; t < cnt; t++) r += tmp[st + t] < key;
      s[st + r] = key;
    }
  }
  __syncwarp();
  return true;
}

// ---------------------------------------------------------------------------
// Register bitonic networks over 32*E keys, blocked layout: lane l holds
// positions E*l .. E*l+E-1.  Strides >= E pair registers of different lanes
// (shuffle), smaller strides pair registers of the same lane.
// ---------------------------------------------------------------------------
// Only the within-lane strides are unrolled (their register indices must be
// static); the cross-lane strides run as a loop, which keeps the live range
// of the network, and so the register count, small.
template <int E>
__device__ __forceinline__ void reg_cross_step(uint64_t (&x)[E], int lane, int size,
                                               int stride) {
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int i = E * lane + j;
    const bool up = (i & size) == 0;
    const bool lower = (i & stride) == 0;
    const uint64_t o = shfl_xor64(x[j], stride / E);
    x[j] = (lower == up) ? umin64(x[j], o) : umax64(x[j], o);
  }
}

template <int E>
__device__ __forceinline__ void reg_inner_steps(uint64_t (&x)[E], int lane, int size) {
#pragma unroll
  for (int stride = E / 2; stride > 0; stride >>= 1) {
    if (stride < size) {
#pragma unroll
      for (int j = 0; j < E; j++) {
        if ((j & stride) == 0) {
          const int j2 = j | stride;
          const bool up = ((E * lane + j) & size) == 0;
          const uint64_t a = x[j], b = x[j2];
          const bool sw = (a > b) == up;
          x[j] = sw ? b : a;
          x[j2] = sw ? a : b;
        }
      }
    }
  }
}

template <int E>
__device__ __forceinline__ void reg_bitonic_sort(uint64_t (&x)[E], int lane) {
  constexpr int L = 32 * E;
#pragma unroll 1
  for (int size = 2; size <= L; size <<= 1) {
#pragma unroll 1
    for (int stride = size >> 1; stride >= E; stride >>= 1)
      reg_cross_step<E>(x, lane, size, stride);
    reg_inner_steps<E>(x, lane, size);
  }
}

// Sorts a bitonic sequence ascending (every comparison ascending: size = 2L).
template <int E>
__device__ __forceinline__ void reg_bitonic_merge(uint64_t (&x)[E], int lane) {
  constexpr int L = 32 * E;
#pragma unroll 1
  for (int stride = L >> 1; stride >= E; stride >>= 1)
    reg_cross_step<E>(x, lane, 2 * L, stride);
  reg_inner_steps<E>(x, lane, 2 * L);
}

// Bitonic sort of n keys in shared memory (n a power of two), ascending, by
// one warp.
__device__ __forceinline__ void smem_bitonic_sort_rt(uint64_t *s, int n, int lane) {
#pragma unroll 1
  for (int size = 2; size <= n; size <<= 1) {
#pragma unroll 1
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll 1
      for (int t = lane; t < n / 2; t += 32) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const uint64_t a = s[i], b = s[j];
        if ((a > b) == up) {
          s[i] = b;
          s[j] = a;
        }
      }
      __syncwarp();
    }
  }
}

}  // namespace knnsweet
