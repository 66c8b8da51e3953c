// common.cuh -- shared device/host helpers of libknnsweet.
//
// Ordering key of a candidate neighbour: the 64-bit word
//     (float bits of the FP32 squared distance) << 32 | reference index.
// Squared distances are non-negative, so their IEEE bit patterns order like
// the values, and the word orders pairs by (distance, index): ties at equal
// distance go to the lower index.  The reference ranks by the square-rooted
// distance with strict-less insertion (src/knnjoin.cu:815-820), which keeps
// whichever tied point it visited first; the index tie-break makes the
// result deterministic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/knnsweet.h"

namespace knnsweet {

constexpr uint64_t kKeyMax = ~0ull;
constexpr unsigned kFull = 0xffffffffu;

__host__ __device__ __forceinline__ uint64_t make_key(float d2, int32_t idx) {
#ifdef __CUDA_ARCH__
  return ((uint64_t)__float_as_uint(d2) << 32) | (uint32_t)idx;
#else
  uint32_t b;
  memcpy(&b, &d2, 4);
  return ((uint64_t)b << 32) | (uint32_t)idx;
#endif
}

__device__ __forceinline__ float key_d2(uint64_t key) {
  return __uint_as_float((uint32_t)(key >> 32));
}
__device__ __forceinline__ int32_t key_idx(uint64_t key) {
  return (int32_t)(uint32_t)(key & 0xffffffffu);
}

// Relative slack that covers FP32 rounding in the distances entering a
// triangle-inequality bound: every computed distance is within (d+4) units
// of 2^-24 of its exact value; bounds are widened by 4x that.
__host__ __device__ __forceinline__ float bound_tol(int d) {
  return (float)(4 * d + 16) * 5.9604645e-8f;
}

// FP32 rounding band of a k-th squared distance Dk.  A squared distance
// computed in FP32 (one rounding per difference, the square fused into an
// fma accumulating non-negative terms in dimension order) is within (d + 2)
// units of 2^-24 (relative) of the exact value of the same FP32 inputs.  So
// a point whose FP32 value lies above band_hi(Dk) is farther, exactly and in
// FP64, than every point at or below Dk, and a point below band_lo(Dk) is
// nearer than every point at or above Dk: only points inside the band can
// rank differently in FP32 and in FP64.  The half-width (2d + 12) units covers
// both values' errors with 8 units to spare for FP64 rounding and the band's
// own arithmetic (rounded outward).
__device__ __forceinline__ float band_hi(float D, int d) {
  return __fmul_ru(D, __fadd_ru(1.0f, (float)(2 * d + 12) * 5.9604645e-8f));
}
__device__ __forceinline__ float band_lo(float D, int d) {
  return __fmul_rd(D, __fsub_rd(1.0f, (float)(2 * d + 12) * 5.9604645e-8f));
}

// FP64 squared distance of the first d coordinates of two rows, in dimension
// order, each product and sum rounded separately -- the arithmetic of the
// FP64 brute-force join the results are checked against.
__device__ __forceinline__ double dist2_f64(const float *__restrict__ a,
                                            const float *__restrict__ b, int d) {
  double acc = 0.0;
  for (int c = 0; c < d; c++) {
    const double t = __dsub_rn((double)a[c], (double)b[c]);
    acc = __dadd_rn(acc, __dmul_rn(t, t));
  }
  return acc;
}

// (FP64 squared distance, index) order: ties go to the lower index.
__device__ __forceinline__ bool f64_key_less(double da, int32_t ia, double db, int32_t ib) {
  return da < db || (da == db && ia < ib);
}

// FP32 squared distance of two padded rows of DP4 float4 (pad lanes are 0 in
// both rows, so they add exactly 0), summed in dimension order with fma.
template <int DP4>
__device__ __forceinline__ float dist2_rows(const float4 (&a)[DP4],
                                           const float4 *__restrict__ b) {
  float acc = 0.0f;
#pragma unroll
  for (int c = 0; c < DP4; c++) {
    float4 v = b[c];
    float t;
    t = __fsub_rn(a[c].x, v.x); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(a[c].y, v.y); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(a[c].z, v.z); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(a[c].w, v.w); acc = __fmaf_rn(t, t, acc);
  }
  return acc;
}

// Same on two rows in memory with a runtime chunk count.
__device__ __forceinline__ float dist2_rows_rt(const float4 *__restrict__ a,
                                               const float4 *__restrict__ b,
                                               int dp4) {
  float acc = 0.0f;
  for (int c = 0; c < dp4; c++) {
    float4 u = a[c];
    float4 v = b[c];
    float t;
    t = __fsub_rn(u.x, v.x); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.y, v.y); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.z, v.z); acc = __fmaf_rn(t, t, acc);
    t = __fsub_rn(u.w, v.w); acc = __fmaf_rn(t, t, acc);
  }
  return acc;
}

// Warp-cooperative lower bound: first position p in [0, n) of the ascending
// array a with a[p] >= v (n if none).  32-ary search: each round the lanes
// sample 32 evenly spaced positions and a ballot brackets the answer, so a
// list of a few thousand members needs two dependent loads instead of ~11.
// Must be called by all 32 lanes with the same arguments.
__device__ __forceinline__ int warp_lower_bound(const float *__restrict__ a,
                                                int n, float v, int lane) {
  int lo = 0, hi = n;  // answer in [lo, hi]
  while (hi - lo > 32) {
    int step = (hi - lo + 31) >> 5;
    int p = lo + (lane + 1) * step - 1;
    bool lt = (p < hi) && (a[p] < v);
    unsigned b = __ballot_sync(kFull, lt);
    int c = __popc(b);
    int nlo = lo + c * step;
    int nhi = lo + (c + 1) * step - 1;  // a[nhi] >= v if nhi < hi
    lo = nlo;
    hi = nhi < hi ? nhi : hi;
  }
  int p = lo + lane;
  bool lt = (p < hi) && (a[p] < v);
  return lo + __popc(__ballot_sync(kFull, lt));
}

// A start for a walk up a sorted array towards the first a[i] >= v: a
// position lo with a[i] < v for every i < lo and that first element at most
// 31 places further on.  The 32-ary search of warp_lower_bound without its
// last level, which saves a dependent load round trip; the walk's own range
// test skips the few elements below v.
__device__ __forceinline__ int warp_lower_bound_coarse(const float *__restrict__ a, int n,
                                                       float v, int lane) {
  int lo = 0, hi = n;
  while (hi - lo > 32) {
    const int step = (hi - lo + 31) >> 5;
    const int p = lo + (lane + 1) * step - 1;
    const int c = __popc(__ballot_sync(kFull, (p < hi) && (a[p] < v)));
    if (step <= 32) return lo + c * step;
    const int nhi = lo + (c + 1) * step - 1;
    lo += c * step;
    hi = nhi < hi ? nhi : hi;
  }
  return lo;
}

// Per-thread last-error text (the C ABI never exits the process).
void set_error(const char *fmt, ...);
std::string &error_buffer();

// Per-thread count of kernels enqueued by the current call (reported in
// knn_stats.kernels_launched); every launch site ends in KNN_LAUNCH_CHECK.
int &launch_counter();
// The per-device stream-ordered pool the library draws its scratch from.
int scratch_pool(cudaMemPool_t *out);

}  // namespace knnsweet

#define KNN_CUDA_TRY(call)                                                   \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      ::knnsweet::set_error("%s failed: %s (%s:%d)", #call,                  \
                            cudaGetErrorString(e_), __FILE__, __LINE__);     \
      return e_ == cudaErrorMemoryAllocation ? KNN_ENOMEM : KNN_ECUDA;       \
    }                                                                        \
  } while (0)

#define KNN_LAUNCH_CHECK()                                                   \
  do {                                                                       \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) {                                                 \
      ::knnsweet::set_error("kernel launch failed: %s (%s:%d)",              \
                            cudaGetErrorString(e_), __FILE__, __LINE__);     \
      return KNN_ECUDA;                                                      \
    }                                                                        \
    ++::knnsweet::launch_counter();                                          \
  } while (0)
