// batched.cu -- the join over many independent point clouds in one call
// (knn_join_batched_device).  The reference joins one pair of point sets per
// process; running it per cloud costs a whole pipeline (and for clouds under
// 13,312 points its tpq > 1 path, src/knnjoin.cu:1103-1127) per cloud.
//
// Here every stage runs once for all clouds:
//   - representatives per cloud: R_c = alpha * sqrt(n_c), alpha picked per
//     cloud-size bucket by the autotuner below; the draw uses a counter-based
//     hash (SplitMix64 of seed, cloud, trial, slot) on the device instead of
//     the host glibc sequence, which would mean millions of values to upload;
//     the best of `rep_trials` draws by pairwise spread, as the single join;
//   - every point is assigned to its own cloud's nearest representative;
//   - one global radix sort on (global cluster id, distance) lays all clouds'
//     clusters out contiguously (clusters of a cloud are consecutive ids);
//   - per query cluster the k-th bound and the candidate list are computed
//     over its own cloud's reference clusters only (variable-length lists);
//   - the shared scan kernel runs over all queries of all clouds, with
//     indices written relative to the start of each reference cloud.
// No host synchronisation between stages: the call can be captured in a CUDA
// graph (after the autotuner, which synchronises, has run once).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "bounds.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace knnsweet {

namespace {

constexpr int kMaxCloudReps = 2048;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// Cloud of a global index given ascending offsets off[0..ncloud]: largest c
// with off[c] <= i.
template <class T>
__device__ __forceinline__ int cloud_of(const T *off, int ncloud, int64_t i) {
  int lo = 0, hi = ncloud - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((int64_t)off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// cand[trials * roff[c] + t * R_c + i]: candidate rows (global) of cloud c.
__global__ void batched_draw_kernel(const int64_t *__restrict__ poff,
                                    const int32_t *__restrict__ roff, int ncloud, int trials,
                                    uint32_t seed, int32_t *__restrict__ cand) {
  const int64_t total = roff[ncloud];
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int c = cloud_of(roff, ncloud, g);
    const int R = roff[c + 1] - roff[c], i = (int)(g - roff[c]);
    const int64_t n = poff[c + 1] - poff[c];
    for (int t = 0; t < trials; t++) {
      const uint64_t h = splitmix64(((uint64_t)seed << 40) ^ ((uint64_t)c << 20) ^
                                    ((uint64_t)t << 12) ^ splitmix64((uint64_t)i));
      cand[(int64_t)trials * roff[c] + (int64_t)t * R + i] = (int32_t)(poff[c] + (int64_t)(h % (uint64_t)n));
    }
  }
}

// One block per (cloud, trial): wrapping sum over ordered candidate pairs of
// (int) distance, candidates staged in shared memory.
__global__ void __launch_bounds__(256)
    batched_rep_score_kernel(const float4 *__restrict__ rows, int dp4,
                             const int32_t *__restrict__ cand,
                             const int32_t *__restrict__ roff, int trials,
                             uint32_t *__restrict__ score) {
  extern __shared__ float4 srow[];
  __shared__ uint32_t red[8];
  const int c = blockIdx.x, t = blockIdx.y;
  const int R = roff[c + 1] - roff[c];
  const int32_t *cc = cand + (int64_t)trials * roff[c] + (int64_t)t * R;
  for (int e = threadIdx.x; e < R * dp4; e += blockDim.x)
    srow[e] = rows[(int64_t)cc[e / dp4] * dp4 + e % dp4];
  __syncthreads();
  // the pair distance is symmetric bit for bit and zero on the diagonal, so
  // the sum over ordered pairs is twice the sum over i < j (wrapping); a
  // thread takes rows t and R - 1 - t, R - 1 distances in all
  uint32_t sum = 0;
  for (int t = threadIdx.x; t < (R + 1) / 2; t += blockDim.x) {
    const int i1 = t, i2 = R - 1 - t;
    for (int j = i1 + 1; j < R; j++)
      sum += (uint32_t)(int32_t)sqrtf(dist2_rows_rt(srow + i1 * dp4, srow + j * dp4, dp4));
    if (i2 != i1)
      for (int j = i2 + 1; j < R; j++)
        sum += (uint32_t)(int32_t)sqrtf(dist2_rows_rt(srow + i2 * dp4, srow + j * dp4, dp4));
  }
  sum *= 2u;
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += red[w];
    score[(int64_t)c * trials + t] = tot;
  }
}

// One block per cloud: first trial whose score (as float) beats a running
// best starting at 0, then its rows become the cloud's representatives.
__global__ void batched_rep_pick_kernel(const float4 *__restrict__ rows, int dp4,
                                        const int32_t *__restrict__ cand,
                                        const int32_t *__restrict__ roff, int trials,
                                        const uint32_t *__restrict__ score,
                                        float4 *__restrict__ reps) {
  __shared__ int best_s;
  const int c = blockIdx.x;
  const int R = roff[c + 1] - roff[c];
  if (threadIdx.x == 0) {
    float best = 0.0f;
    int bt = 0;
    for (int t = 0; t < trials; t++) {
      const float v = (float)(int32_t)score[(int64_t)c * trials + t];
      if (best < v) {
        best = v;
        bt = t;
      }
    }
    best_s = bt;
  }
  __syncthreads();
  const int32_t *cc = cand + (int64_t)trials * roff[c] + (int64_t)best_s * R;
  for (int e = threadIdx.x; e < R * dp4; e += blockDim.x)
    reps[((int64_t)roff[c] + e / dp4) * dp4 + e % dp4] = rows[(int64_t)cc[e / dp4] * dp4 + e % dp4];
}

// Nearest representative of the point's own cloud (lowest index on ties).
// Block b covers 256 points of cloud c (chunk_off[c] <= b < chunk_off[c+1]).
__global__ void __launch_bounds__(256)
    batched_assign_kernel(const float4 *__restrict__ rows, int dp4,
                          const int64_t *__restrict__ poff, const int32_t *__restrict__ roff,
                          const int32_t *__restrict__ chunk_off, int ncloud,
                          const float4 *__restrict__ reps, int32_t *__restrict__ cl,
                          float *__restrict__ dr) {
  extern __shared__ float4 srep[];
  const int b = blockIdx.x;
  const int c = cloud_of(chunk_off, ncloud, b);
  const int R = roff[c + 1] - roff[c];
  for (int e = threadIdx.x; e < R * dp4; e += blockDim.x)
    srep[e] = reps[(int64_t)roff[c] * dp4 + e];
  __syncthreads();
  const int64_t i = poff[c] + (int64_t)(b - chunk_off[c]) * 256 + threadIdx.x;
  if (i >= poff[c + 1]) return;
  float best = __int_as_float(0x7f7fffff);
  int bi = 0;
  for (int j = 0; j < R; j++) {
    const float v = dist2_rows_rt(rows + i * dp4, srep + j * dp4, dp4);
    if (v < best) {
      best = v;
      bi = j;
    }
  }
  cl[i] = roff[c] + bi;
  dr[i] = sqrtf(best);
}

// Per query cluster: the k-th bound and the candidate list over its own
// cloud's reference clusters.  Representative distances are computed here
// (into shared memory); the list goes to rlist[rl_base[qc] ..].
// dynamic shared memory: rs_pow2 keys + max_rs floats
__global__ void __launch_bounds__(512)
    batched_bounds_kernel(const float4 *__restrict__ qreps, const float4 *__restrict__ sreps,
                          int dp4, const int32_t *__restrict__ q_roff,
                          const int32_t *__restrict__ s_roff,
                          const int64_t *__restrict__ pair_off,
                          const int64_t *__restrict__ r_poff, int ncloud,
                          const int32_t *__restrict__ qoff, const int32_t *__restrict__ soff,
                          const float *__restrict__ sdist, const float *__restrict__ scmax,
                          const float *__restrict__ qrad, int k, int d, int rs_pow2,
                          float *__restrict__ theta0, int32_t *__restrict__ rlist,
                          int32_t *__restrict__ rlen, int64_t *__restrict__ rl_base,
                          int64_t *__restrict__ qc_ref_base) {
  extern __shared__ uint64_t skey[];
  float *dq = reinterpret_cast<float *>(skey + rs_pow2);
  const int qc = blockIdx.x;
  const int c = cloud_of(q_roff, ncloud, qc);
  const int sb = s_roff[c], Rs_loc = s_roff[c + 1] - sb;
  const int64_t base = pair_off[c] + (int64_t)(qc - q_roff[c]) * Rs_loc;
  if (threadIdx.x == 0) {
    rl_base[qc] = base;
    qc_ref_base[qc] = r_poff[c];
  }
  if (qoff[qc + 1] == qoff[qc] || Rs_loc == 0) {
    if (threadIdx.x == 0) {
      theta0[qc] = 0.0f;
      rlen[qc] = 0;
    }
    return;
  }
  for (int j = threadIdx.x; j < Rs_loc; j += blockDim.x)
    dq[j] = sqrtf(dist2_rows_rt(qreps + (int64_t)qc * dp4, sreps + (int64_t)(sb + j) * dp4, dp4));
  __syncthreads();
  bounds_filter_block(dq, Rs_loc, soff + sb, sdist, scmax + sb, qrad[qc], k, d, rs_pow2, sb,
                      skey, theta0 + qc, rlist + base, rlen + qc);
}

// The same per query cluster, one warp each (clouds with at most a few
// hundred representatives): kBoundsWarps warps per block, each with its own
// `per_warp` bytes of dynamic shared memory (rs_pow2 keys, then max_rs floats).
constexpr int kBoundsWarps = 8;

__global__ void __launch_bounds__(kBoundsWarps * 32)
    batched_bounds_warp_kernel(const float4 *__restrict__ qreps, const float4 *__restrict__ sreps,
                               int dp4, const int32_t *__restrict__ q_roff,
                               const int32_t *__restrict__ s_roff,
                               const int64_t *__restrict__ pair_off,
                               const int64_t *__restrict__ r_poff, int ncloud, int nqc,
                               const int32_t *__restrict__ qoff, const int32_t *__restrict__ soff,
                               const float *__restrict__ sdist, const float *__restrict__ scmax,
                               const float *__restrict__ qrad, int k, int d, int rs_pow2,
                               int per_warp, float *__restrict__ theta0,
                               int32_t *__restrict__ rlist, int32_t *__restrict__ rlen,
                               int64_t *__restrict__ rl_base, int64_t *__restrict__ qc_ref_base) {
  extern __shared__ __align__(16) unsigned char wsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qc = blockIdx.x * kBoundsWarps + warp;
  if (qc >= nqc) return;  // whole warps only; no block barrier follows
  uint64_t *skey = reinterpret_cast<uint64_t *>(wsm + (size_t)warp * per_warp);
  float *dq = reinterpret_cast<float *>(skey + rs_pow2);
  const int c = cloud_of(q_roff, ncloud, qc);
  const int sb = s_roff[c], Rs_loc = s_roff[c + 1] - sb;
  const int64_t base = pair_off[c] + (int64_t)(qc - q_roff[c]) * Rs_loc;
  if (lane == 0) {
    rl_base[qc] = base;
    qc_ref_base[qc] = r_poff[c];
  }
  if (qoff[qc + 1] == qoff[qc] || Rs_loc == 0) {
    if (lane == 0) {
      theta0[qc] = 0.0f;
      rlen[qc] = 0;
    }
    return;
  }
  for (int j = lane; j < Rs_loc; j += 32)
    dq[j] = sqrtf(dist2_rows_rt(qreps + (int64_t)qc * dp4, sreps + (int64_t)(sb + j) * dp4, dp4));
  __syncwarp();
  bounds_filter_warp(dq, Rs_loc, soff + sb, sdist, scmax + sb, qrad[qc], k, d, sb, skey,
                     theta0 + qc, rlist + base, rlen + qc, lane);
}

__global__ void batched_fill_empty_kernel(int32_t *idx, float *dist, int64_t count) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    idx[t] = -1;
    dist[t] = __int_as_float(0x7f800000);
  }
}

#define KNN_TRY(expr)              \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != KNN_OK) return rc_; \
  } while (0)

// Stream-ordered scratch from the library's per-device pool, released on
// the same stream when the arena goes out of scope.
class BatchArena {
 public:
  explicit BatchArena(cudaStream_t s) : s_(s) {}
  ~BatchArena() {
    for (void *p : ptrs_) cudaFreeAsync(p, s_);
  }
  BatchArena(const BatchArena &) = delete;
  BatchArena &operator=(const BatchArena &) = delete;
  template <class T>
  int alloc(T **out, size_t count) {
    *out = nullptr;
    if (!pool_) KNN_TRY(scratch_pool(&pool_));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, (count ? count : 1) * sizeof(T), pool_, s_);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation failed: %s", cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? KNN_ENOMEM : KNN_ECUDA;
    }
    ptrs_.push_back(p);
    *out = static_cast<T *>(p);
    return KNN_OK;
  }

 private:
  cudaStream_t s_;
  cudaMemPool_t pool_ = nullptr;
  std::vector<void *> ptrs_;
};

// Host arrays reach the device as kernel parameters (no pageable copy, so
// the call stays capturable).
struct U32Chunk {
  int32_t count;
  uint32_t v[8000];
};
__global__ void batched_upload_kernel(uint32_t *__restrict__ dst, const U32Chunk c) {
  for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[i] = c.v[i];
}
int upload_words(const void *src, size_t words, void *dst, cudaStream_t s) {
  U32Chunk c;
  const uint32_t *w = static_cast<const uint32_t *>(src);
  for (size_t base = 0; base < words; base += 8000) {
    const size_t cnt = std::min<size_t>(8000, words - base);
    c.count = (int32_t)cnt;
    memcpy(c.v, w + base, cnt * sizeof(uint32_t));
    batched_upload_kernel<<<1, 256, 0, s>>>(static_cast<uint32_t *>(dst) + base, c);
    KNN_LAUNCH_CHECK();
  }
  return KNN_OK;
}

// One side (query or reference clouds) clustered.
struct BatchSide {
  int64_t total = 0;
  int Rtot = 0, maxR = 0;
  const float4 *rows = nullptr;
  int64_t *poff = nullptr;  // device, ncloud + 1
  int32_t *roff = nullptr;  // device, ncloud + 1
  float4 *reps = nullptr;
  uint64_t *skeys = nullptr;
  int32_t *perm = nullptr;
  int32_t *off = nullptr;   // Rtot + 1
};

int cluster_side(BatchArena &ar, const float *pts, const int64_t *off_h, int ncloud, int d,
                 int dp4, const std::vector<int32_t> &R_h, uint32_t seed, int trials,
                 cudaStream_t s, BatchSide *b) {
  b->total = off_h[ncloud];
  std::vector<int32_t> roff_h(ncloud + 1, 0), chunk_h(ncloud + 1, 0);
  for (int c = 0; c < ncloud; c++) {
    roff_h[c + 1] = roff_h[c] + R_h[c];
    chunk_h[c + 1] = chunk_h[c] + (int32_t)((off_h[c + 1] - off_h[c] + 255) / 256);
    b->maxR = std::max(b->maxR, R_h[c]);
  }
  b->Rtot = roff_h[ncloud];
  int32_t *chunk = nullptr;
  KNN_TRY(ar.alloc(&b->poff, (size_t)ncloud + 1));
  KNN_TRY(ar.alloc(&b->roff, (size_t)ncloud + 1));
  KNN_TRY(ar.alloc(&chunk, (size_t)ncloud + 1));
  KNN_TRY(upload_words(off_h, 2 * (size_t)(ncloud + 1), b->poff, s));
  KNN_TRY(upload_words(roff_h.data(), (size_t)ncloud + 1, b->roff, s));
  KNN_TRY(upload_words(chunk_h.data(), (size_t)ncloud + 1, chunk, s));
  // rows as float4
  if (dp4 * 4 == d && (reinterpret_cast<uintptr_t>(pts) & 15) == 0) {
    b->rows = reinterpret_cast<const float4 *>(pts);
  } else {
    float4 *p;
    KNN_TRY(ar.alloc(&p, (size_t)b->total * dp4));
    KNN_TRY(launch_pack_rows(pts, b->total, d, dp4, p, s));
    b->rows = p;
  }
  // representatives: draw, score, pick
  int32_t *cand;
  uint32_t *score;
  KNN_TRY(ar.alloc(&cand, (size_t)trials * b->Rtot));
  KNN_TRY(ar.alloc(&score, (size_t)trials * ncloud));
  KNN_TRY(ar.alloc(&b->reps, (size_t)b->Rtot * dp4));
  batched_draw_kernel<<<148 * 8, 256, 0, s>>>(b->poff, b->roff, ncloud, trials, seed, cand);
  KNN_LAUNCH_CHECK();
  const size_t srow_bytes = (size_t)b->maxR * dp4 * sizeof(float4);
  if (srow_bytes > 48 * 1024) {
    KNN_CUDA_TRY(cudaFuncSetAttribute(batched_rep_score_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)srow_bytes));
    KNN_CUDA_TRY(cudaFuncSetAttribute(batched_assign_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)srow_bytes));
  }
  batched_rep_score_kernel<<<dim3(ncloud, trials), 256, srow_bytes, s>>>(b->rows, dp4, cand,
                                                                        b->roff, trials, score);
  KNN_LAUNCH_CHECK();
  batched_rep_pick_kernel<<<ncloud, 256, 0, s>>>(b->rows, dp4, cand, b->roff, trials, score,
                                                 b->reps);
  KNN_LAUNCH_CHECK();
  // assignment, one global sort, offsets
  int32_t *cl;
  float *dr;
  KNN_TRY(ar.alloc(&cl, (size_t)b->total));
  KNN_TRY(ar.alloc(&dr, (size_t)b->total));
  if (chunk_h[ncloud] > 0) {
    batched_assign_kernel<<<chunk_h[ncloud], 256, srow_bytes, s>>>(
        b->rows, dp4, b->poff, b->roff, chunk, ncloud, b->reps, cl, dr);
    KNN_LAUNCH_CHECK();
  }
  uint64_t *keys;
  int32_t *vals;
  KNN_TRY(ar.alloc(&keys, (size_t)b->total));
  KNN_TRY(ar.alloc(&vals, (size_t)b->total));
  KNN_TRY(ar.alloc(&b->skeys, (size_t)b->total));
  KNN_TRY(ar.alloc(&b->perm, (size_t)b->total));
  const size_t temp_bytes = cluster_sort_temp_bytes(b->total, std::max(b->Rtot, 1));
  unsigned char *temp;
  KNN_TRY(ar.alloc(&temp, temp_bytes));
  KNN_TRY(launch_cluster_sort(cl, dr, b->total, std::max(b->Rtot, 1), keys, vals, b->skeys,
                              b->perm, temp, temp_bytes, s));
  KNN_TRY(ar.alloc(&b->off, (size_t)b->Rtot + 1));
  KNN_TRY(launch_cluster_offsets(b->skeys, b->total, b->Rtot, b->off, s));
  return KNN_OK;
}

// Representatives of a cloud of n points; at most kMaxCloudReps, and few
// enough that one cloud's representative rows fit in shared memory.
int reps_for_cloud(int64_t n, float alpha, int dp4) {
  if (n <= 0) return 0;
  const int cap = std::min(kMaxCloudReps, 12288 / dp4);
  const int64_t r = (int64_t)std::floor(alpha * std::sqrt((double)n) + 0.5);
  return (int)std::max<int64_t>(1, std::min<int64_t>({r, n, (int64_t)cap}));
}

int size_bucket(int64_t n) {
  int b = 0;
  while ((int64_t)1 << (b + 1) <= n) b++;
  return b;
}

int batched_impl(const float *q, const int64_t *qoff_h, const float *r, const int64_t *roff_h,
                 int ncloud, int d, int k, int32_t *out_idx, float *out_dist,
                 const knn_options &o, const std::vector<float> &alpha_of_cloud,
                 knn_stats *st, cudaStream_t s) {
  const int64_t m = qoff_h[ncloud];
  const bool self = q == r && std::equal(qoff_h, qoff_h + ncloud + 1, roff_h);
  int dev = 0, num_sms = 148;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  KNN_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  const int dp4r = (d + 3) / 4;
  int dp4 = 1;
  while (dp4 < dp4r) dp4 <<= 1;
  std::vector<int32_t> Rs_h(ncloud), Rq_h(ncloud);
  for (int c = 0; c < ncloud; c++) {
    Rs_h[c] = reps_for_cloud(roff_h[c + 1] - roff_h[c], alpha_of_cloud[c], dp4);
    Rq_h[c] = self ? Rs_h[c] : reps_for_cloud(qoff_h[c + 1] - qoff_h[c], alpha_of_cloud[c], dp4);
  }
  cudaEvent_t ev[3] = {};
  if (st) {
    for (auto &e : ev) KNN_CUDA_TRY(cudaEventCreate(&e));
    KNN_CUDA_TRY(cudaEventRecord(ev[0], s));
  }
  int rc = KNN_OK;
  {
    BatchArena ar(s);
    unsigned long long *ctr = nullptr;
    auto body = [&]() -> int {
      // [0] scan work counter, [1 ..] scan statistics, then the count of
      // queries left to the band kernel
      constexpr int kCtr = 4 + kScanCounters;  // + the two sides' exactness flags
      KNN_TRY(ar.alloc(&ctr, kCtr));
      KNN_CUDA_TRY(cudaMemsetAsync(ctr, 0, kCtr * sizeof(unsigned long long), s));
      if (roff_h[ncloud] == 0) {  // no reference points in any cloud
        batched_fill_empty_kernel<<<148, 256, 0, s>>>(out_idx, out_dist, m * (int64_t)k);
        KNN_LAUNCH_CHECK();
        return KNN_OK;
      }
      BatchSide S, Q;
      KNN_TRY(cluster_side(ar, r, roff_h, ncloud, d, dp4, Rs_h, o.seed, o.rep_trials, s, &S));
      const int64_t n = S.total;
      float4 *srows;
      float *sdist, *cmin, *cmax;
      int32_t *sidx;
      KNN_TRY(ar.alloc(&srows, (size_t)n * dp4));
      KNN_TRY(ar.alloc(&sdist, (size_t)n));
      KNN_TRY(ar.alloc(&sidx, (size_t)n));
      KNN_TRY(ar.alloc(&cmin, (size_t)S.Rtot + 1));
      KNN_TRY(ar.alloc(&cmax, (size_t)S.Rtot + 1));
      const bool idx_in_row = 4 * dp4 > d;
      KNN_TRY(launch_cluster_layout(S.skeys, S.perm, n, S.rows, dp4, idx_in_row, srows, sdist,
                                    sidx, s));
      KNN_TRY(launch_cluster_minmax(S.off, sdist, S.Rtot, cmin, cmax, s));
      if (self) {
        Q = S;
      } else {
        KNN_TRY(cluster_side(ar, q, qoff_h, ncloud, d, dp4, Rq_h, o.seed, o.rep_trials, s, &Q));
      }
      // per-cloud offsets of the candidate lists
      std::vector<int64_t> pair_h(ncloud + 1, 0);
      for (int c = 0; c < ncloud; c++) pair_h[c + 1] = pair_h[c] + (int64_t)Rq_h[c] * Rs_h[c];
      int64_t *pair_off, *rl_base, *qc_ref_base;
      KNN_TRY(ar.alloc(&pair_off, (size_t)ncloud + 1));
      KNN_TRY(upload_words(pair_h.data(), 2 * (size_t)(ncloud + 1), pair_off, s));
      float *qrad, *theta0;
      int32_t *slot_cl, *rlist, *rlen;
      KNN_TRY(ar.alloc(&qrad, (size_t)Q.Rtot + 1));
      KNN_TRY(ar.alloc(&slot_cl, (size_t)m + 1));
      KNN_TRY(launch_query_clusters(Q.skeys, Q.off, m, Q.Rtot, qrad, slot_cl, s));
      KNN_TRY(ar.alloc(&theta0, (size_t)Q.Rtot + 1));
      KNN_TRY(ar.alloc(&rlen, (size_t)Q.Rtot + 1));
      KNN_TRY(ar.alloc(&rl_base, (size_t)Q.Rtot + 1));
      KNN_TRY(ar.alloc(&qc_ref_base, (size_t)Q.Rtot + 1));
      KNN_TRY(ar.alloc(&rlist, (size_t)std::max<int64_t>(pair_h[ncloud], 1)));
      if (Q.Rtot > 0) {
        int p2 = 1;
        while (p2 < S.maxR) p2 <<= 1;
        const size_t smem = (size_t)p2 * sizeof(uint64_t) + (size_t)S.maxR * sizeof(float);
        // a warp per query cluster while each warp's share of shared memory
        // is small (up to 512 representatives per cloud); a block otherwise
        const int per_warp = (int)((smem + 15) & ~(size_t)15);
        if (per_warp <= 6 * 1024) {
          const size_t wsmem = (size_t)kBoundsWarps * per_warp;
          if (wsmem > 48 * 1024)
            KNN_CUDA_TRY(cudaFuncSetAttribute(batched_bounds_warp_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)wsmem));
          batched_bounds_warp_kernel<<<(unsigned)((Q.Rtot + kBoundsWarps - 1) / kBoundsWarps),
                                       kBoundsWarps * 32, wsmem, s>>>(
              Q.reps, S.reps, dp4, Q.roff, S.roff, pair_off, S.poff, ncloud, (int)Q.Rtot, Q.off,
              S.off, sdist, cmax, qrad, k, d, p2, per_warp, theta0, rlist, rlen, rl_base,
              qc_ref_base);
          KNN_LAUNCH_CHECK();
        } else {
          if (smem > 48 * 1024)
            KNN_CUDA_TRY(cudaFuncSetAttribute(batched_bounds_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
          const int nth = std::min(512, std::max(64, p2 / 2));
          batched_bounds_kernel<<<Q.Rtot, nth, smem, s>>>(
              Q.reps, S.reps, dp4, Q.roff, S.roff, pair_off, S.poff, ncloud, Q.off, S.off,
              sdist, cmax, qrad, k, d, p2, theta0, rlist, rlen, rl_base, qc_ref_base);
          KNN_LAUNCH_CHECK();
        }
      }
      if (st) KNN_CUDA_TRY(cudaEventRecord(ev[1], s));
      ScanArgs a{};
      a.qrows = Q.rows;
      a.qorder = Q.perm;
      a.slot_cl = slot_cl;
      a.m = m;
      a.d = d;
      a.dp4 = dp4;
      a.dp4_tmpl = dp4;
      a.k = k;
      a.idx_in_row = idx_in_row;
      a.squared = (o.flags & KNN_SQUARED_DIST) != 0;
      a.sreps = S.reps;
      a.srows = srows;
      a.sdist = sdist;
      a.sidx = sidx;
      a.soff = S.off;
      a.cmin = cmin;
      a.cmax = cmax;
      a.theta0 = theta0;
      a.qrad = qrad;
      a.qkeys = Q.skeys;
      a.rlist = rlist;
      a.rlen = rlen;
      a.rl_base = rl_base;
      a.qc_ref_base = qc_ref_base;
      a.Rs = S.Rtot;
      a.n_ref = S.total;
      a.rrows = S.rows;
      {
        int *fr = reinterpret_cast<int *>(ctr + 2 + kScanCounters);
        int *fq = reinterpret_cast<int *>(ctr + 3 + kScanCounters);
        KNN_TRY(launch_exact_check(reinterpret_cast<const float *>(S.rows), n * dp4 * 4, d, fr,
                                   s));
        if (!self)
          KNN_TRY(launch_exact_check(reinterpret_cast<const float *>(Q.rows), m * dp4 * 4, d, fq,
                                     s));
        a.inexact_r = fr;
        a.inexact_q = self ? fr : fq;
      }
      a.out_idx = out_idx;
      a.out_dist = out_dist;
      KNN_TRY(ar.alloc(&a.unres_slot, (size_t)m));
      a.unres_count = reinterpret_cast<unsigned *>(ctr + 1 + kScanCounters);
      a.work_counter = ctr;
      a.counters = ctr + 1;
      KNN_TRY(launch_scan(a, num_sms, s));
      if (st) {
        KNN_CUDA_TRY(cudaEventRecord(ev[2], s));
        unsigned long long h[kCtr];
        KNN_CUDA_TRY(cudaMemcpyAsync(h, ctr, sizeof h, cudaMemcpyDeviceToHost, s));
        KNN_CUDA_TRY(cudaStreamSynchronize(s));
        st->dist_evals = (int64_t)h[1];
        st->clusters_visited = (int64_t)h[2];
        st->clusters_pruned = (int64_t)h[3];
        st->topk_candidates = (int64_t)h[4];
        st->topk_merges = (int64_t)h[5];
        st->fp64_rechecks = (int64_t)h[6];
        st->band_queries = (int32_t)h[7];
        int64_t pairs = 0;
        for (int c = 0; c < ncloud; c++)
          pairs += (qoff_h[c + 1] - qoff_h[c]) * (roff_h[c + 1] - roff_h[c]);
        st->pairs_total = pairs;
        st->pairs_pruned = pairs - st->dist_evals;
        st->qreps_used = Q.Rtot;
        st->sreps_used = S.Rtot;
        st->kernels_launched = launch_counter();
        KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_build, ev[0], ev[1]));
        KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_search, ev[1], ev[2]));
        KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_total, ev[0], ev[2]));
      }
      return KNN_OK;
    };
    rc = body();
  }
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

// ---------------------------------------------------------------------------
// Autotuner: representatives per cloud = alpha * sqrt(n_c), alpha chosen per
// cloud-size bucket (powers of two) by timing the batched join on up to 256
// clouds of the bucket with each candidate alpha (one untimed run, then the
// best of two timed runs).  Results are cached per (d, k, bucket) for the
// process.
// ---------------------------------------------------------------------------
constexpr float kAlphaDefault = 1.6f;
constexpr float kAlphaCandidates[] = {0.5f, 1.0f, 1.6f, 2.5f};

struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int create() {
    KNN_CUDA_TRY(cudaEventCreate(&e0));
    KNN_CUDA_TRY(cudaEventCreate(&e1));
    return KNN_OK;
  }
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, bool>, float> g_tuned;

int autotune(const float *q, const int64_t *qoff_h, const float *r, const int64_t *roff_h,
             int ncloud, int d, int k, const knn_options &o, cudaStream_t s,
             std::vector<float> *alpha_of_cloud) {
  const bool self = q == r && std::equal(qoff_h, qoff_h + ncloud + 1, roff_h);
  std::map<int, std::vector<int>> buckets;
  for (int c = 0; c < ncloud; c++) buckets[size_bucket(roff_h[c + 1] - roff_h[c])].push_back(c);
  std::map<int, float> pick;
  for (auto &kv : buckets) {
    const auto key = std::make_tuple(d, k, kv.first, self);
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        pick[kv.first] = it->second;
        continue;
      }
    }
    // sample: up to 256 clouds of the bucket, copied contiguously
    const std::vector<int> &cs = kv.second;
    const int ns = std::min<int>(256, (int)cs.size());
    std::vector<int64_t> so(ns + 1, 0), sq(ns + 1, 0);
    for (int i = 0; i < ns; i++) {
      so[i + 1] = so[i] + (roff_h[cs[i] + 1] - roff_h[cs[i]]);
      sq[i + 1] = sq[i] + (qoff_h[cs[i] + 1] - qoff_h[cs[i]]);
    }
    float best_a = kAlphaDefault;
    {
      BatchArena ar(s);
      float *sr, *sqp, *od;
      int32_t *oi;
      KNN_TRY(ar.alloc(&sr, (size_t)d * so[ns]));
      if (self) sqp = sr;
      else KNN_TRY(ar.alloc(&sqp, (size_t)d * sq[ns]));
      KNN_TRY(ar.alloc(&oi, (size_t)k * sq[ns]));
      KNN_TRY(ar.alloc(&od, (size_t)k * sq[ns]));
      for (int i = 0; i < ns; i++) {
        KNN_CUDA_TRY(cudaMemcpyAsync(sr + so[i] * d, r + roff_h[cs[i]] * d,
                                     sizeof(float) * d * (so[i + 1] - so[i]),
                                     cudaMemcpyDeviceToDevice, s));
        if (!self)
          KNN_CUDA_TRY(cudaMemcpyAsync(sqp + sq[i] * d, q + qoff_h[cs[i]] * d,
                                       sizeof(float) * d * (sq[i + 1] - sq[i]),
                                       cudaMemcpyDeviceToDevice, s));
      }
      EventPair ev;
      KNN_TRY(ev.create());
      float best_t = 1e30f;
      for (float a : kAlphaCandidates) {
        std::vector<float> al(ns, a);
        float tmin = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
          KNN_CUDA_TRY(cudaEventRecord(ev.e0, s));
          KNN_TRY(batched_impl(sqp, sq.data(), sr, so.data(), ns, d, k, oi, od, o, al, nullptr,
                               s));
          KNN_CUDA_TRY(cudaEventRecord(ev.e1, s));
          KNN_CUDA_TRY(cudaEventSynchronize(ev.e1));
          float ms = 0.0f;
          KNN_CUDA_TRY(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
          if (rep > 0) tmin = std::min(tmin, ms);
        }
        if (tmin < best_t) {
          best_t = tmin;
          best_a = a;
        }
      }
    }
    pick[kv.first] = best_a;
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tuned[key] = best_a;
  }
  for (int c = 0; c < ncloud; c++)
    (*alpha_of_cloud)[c] = pick[size_bucket(roff_h[c + 1] - roff_h[c])];
  return KNN_OK;
}

}  // namespace
}  // namespace knnsweet

using namespace knnsweet;

extern "C" int knn_join_batched_device(const float *q, const int64_t *q_offsets,
                                       const float *r, const int64_t *r_offsets,
                                       int32_t ncloud, int32_t d, int32_t k, int32_t *out_idx,
                                       float *out_dist, const knn_options *opt,
                                       knn_stats *st, void *stream) {
  error_buffer().clear();
  launch_counter() = 0;
  knn_options o;
  knn_default_options(&o);
  if (opt) o = *opt;
  if (st) memset(st, 0, sizeof *st);
  if (ncloud < 0 || d <= 0 || d > 32 || k <= 0 || k > 256 || !q_offsets || !r_offsets) {
    set_error("batched join: need ncloud >= 0, 1 <= d <= 32, 1 <= k <= 256, host offsets");
    return KNN_EINVAL;
  }
  if (o.rep_trials <= 0 || o.rep_trials > 1000 ||
      (o.flags & ~(KNN_SQUARED_DIST | KNN_NO_TENSOR_CORES)) != 0) {
    set_error("batched join: bad options");
    return KNN_EINVAL;
  }
  if (ncloud == 0) return KNN_OK;
  for (int c = 0; c < ncloud; c++) {
    if (q_offsets[c + 1] < q_offsets[c] || r_offsets[c + 1] < r_offsets[c]) {
      set_error("batched join: offsets must be non-decreasing");
      return KNN_EINVAL;
    }
  }
  if (q_offsets[0] != 0 || r_offsets[0] != 0 || r_offsets[ncloud] > INT32_MAX ||
      q_offsets[ncloud] > INT32_MAX) {
    set_error("batched join: offsets must start at 0 and stay below 2^31");
    return KNN_EINVAL;
  }
  if (q_offsets[ncloud] == 0) return KNN_OK;
  if (!q || !r || !out_idx || !out_dist) {
    set_error("batched join: null pointer argument");
    return KNN_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<float> alpha(ncloud, kAlphaDefault);
  if (o.autotune) {
    int rc = autotune(q, q_offsets, r, r_offsets, ncloud, d, k, o, s, &alpha);
    if (rc != KNN_OK) return rc;
  }
  launch_counter() = 0;
  return batched_impl(q, q_offsets, r, r_offsets, ncloud, d, k, out_idx, out_dist, o, alpha, st,
                      s);
}

// Host-buffer form (the reference's per-run host arrays, src/knnjoin.cu:
// 1003-1033, for many runs at once): copies the clouds in on a stream of its
// own, joins them with knn_join_batched_device and copies the result back.
extern "C" int knn_join_batched(const float *q, const int64_t *q_offsets, const float *r,
                                const int64_t *r_offsets, int32_t ncloud, int32_t d, int32_t k,
                                int32_t *out_idx, float *out_dist, const knn_options *opt,
                                knn_stats *st) {
  error_buffer().clear();
  if (st) memset(st, 0, sizeof *st);
  if (ncloud < 0 || d <= 0 || k <= 0 || !q_offsets || !r_offsets) {
    set_error("batched join: need ncloud >= 0, d > 0, k > 0 and host offsets");
    return KNN_EINVAL;
  }
  if (ncloud == 0) return KNN_OK;
  const int64_t m = q_offsets[ncloud], n = r_offsets[ncloud];
  if (m < 0 || n < 0 || m > INT32_MAX || n > INT32_MAX) {
    set_error("batched join: offsets must stay in [0, 2^31)");
    return KNN_EINVAL;
  }
  if (m == 0) {
    // the device entry point validates the rest; no buffers are touched
    return knn_join_batched_device(nullptr, q_offsets, nullptr, r_offsets, ncloud, d, k, nullptr,
                                   nullptr, opt, st, nullptr);
  }
  if (!q || (!r && n > 0) || !out_idx || !out_dist) {
    set_error("batched join: null pointer argument");
    return KNN_EINVAL;
  }
  const bool self = q == r && std::equal(q_offsets, q_offsets + ncloud + 1, r_offsets);
  cudaStream_t s, cs;
  {
    const int rc = host_streams(&s, &cs);
    if (rc != KNN_OK) return rc;
  }
  int rc = KNN_OK;
  {
    BatchArena ar(s);
    float *dq = nullptr, *dr = nullptr, *dd = nullptr;
    int32_t *di = nullptr;
    rc = ar.alloc(&dq, (size_t)m * d);
    if (rc == KNN_OK && !self) rc = ar.alloc(&dr, (size_t)n * d);
    if (rc == KNN_OK) rc = ar.alloc(&di, (size_t)m * k);
    if (rc == KNN_OK) rc = ar.alloc(&dd, (size_t)m * k);
    if (self) dr = dq;
    cudaError_t e = cudaSuccess;
    if (rc == KNN_OK) e = cudaMemcpyAsync(dq, q, sizeof(float) * m * d, cudaMemcpyHostToDevice, s);
    if (rc == KNN_OK && e == cudaSuccess && !self && n > 0)
      e = cudaMemcpyAsync(dr, r, sizeof(float) * n * d, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      set_error("host-to-device copy failed: %s", cudaGetErrorString(e));
      rc = KNN_ECUDA;
    }
    if (rc == KNN_OK)
      rc = knn_join_batched_device(dq, q_offsets, dr, r_offsets, ncloud, d, k, di, dd, opt, st,
                                   s);
    if (rc == KNN_OK) {
      e = cudaMemcpyAsync(out_idx, di, sizeof(int32_t) * m * k, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_dist, dd, sizeof(float) * m * k, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) {
        set_error("device-to-host copy failed: %s", cudaGetErrorString(e));
        rc = KNN_ECUDA;
      }
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess && rc == KNN_OK) {
    set_error("batched join failed on the device: %s", cudaGetErrorString(e));
    rc = KNN_ECUDA;
  }
  return rc;
}
