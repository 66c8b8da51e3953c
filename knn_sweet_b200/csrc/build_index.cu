// build_index.cu -- device-side index build of the pruned kNN join.
//
// Stages (each replaces the reference code cited on it):
//   pack_rows_kernel       row-major input -> padded float4 rows
//   rep_score_kernel       spread score of each random representative draw
//   rep_pick_kernel        first best draw -> representative rows
//   assign_kernel<DP4>     nearest representative + distance per point
//   cluster_keys_kernel    (cluster, distance) sort keys
//   cluster_layout_kernel  cluster-contiguous, distance-sorted copy of the rows
//   cluster_bounds_kernel  cluster offsets, min/max member distance
//   rep_dist_kernel        representative-to-representative distances
//   bounds_filter_kernel   per query cluster: k-th upper bound + surviving
//                          reference clusters sorted by rep-rep distance
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "bounds.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace knnsweet {

// ---------------------------------------------------------------------------
// Row packing: n x d row-major floats -> n x dp4 float4 (zero padded).
// ---------------------------------------------------------------------------
__global__ void pack_rows_kernel(const float *__restrict__ src, int64_t n,
                                 int d, int dp4, float4 *__restrict__ dst) {
  int64_t total = n * dp4;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t row = t / dp4;
    int c = (int)(t - row * dp4);
    const float *s = src + row * d + 4 * c;
    int rem = d - 4 * c;  // <= 0 for chunks past ceil(d/4) (power-of-2 width)
    float4 v;
    v.x = rem > 0 ? s[0] : 0.0f;
    v.y = rem > 1 ? s[1] : 0.0f;
    v.z = rem > 2 ? s[2] : 0.0f;
    v.w = rem > 3 ? s[3] : 0.0f;
    dst[t] = v;
  }
}

// ---------------------------------------------------------------------------
// Representative draw (src/knnjoin.cu:125-154, host draw 195-239).
// cand[t * R + i] are row indices drawn on the host with the glibc generator.
// score[t] = wrapping int32 sum over ordered pairs (i, j) of (int)dist.
// Tiled: a block owns (16 TB) x (16 TB) candidate pairs of one trial; rows are
// staged through shared memory 32 floats at a time and every thread
// accumulates TB x TB pairs (i = i0 + ty + 16a, j = j0 + tx + 16b), each
// summed in dimension order with fma, exactly as the one-pair distance would
// be.  The pair distance is symmetric bit for bit (fsub(a, b) = -fsub(b, a)
// and squaring drops the sign), so only the tiles on and above the diagonal
// run, and an off-diagonal tile counts twice (wrapping, like the sum).
// grid: (nb (nb + 1) / 2 tiles, 1, trials), nb = ceil(R / 16TB), 256 threads
// ---------------------------------------------------------------------------
template <int TB>
__global__ void __launch_bounds__(256)
    rep_score_kernel(const float4 *__restrict__ rows, int dp4,
                     const int32_t *__restrict__ cand, int R,
                     uint32_t *__restrict__ score) {
  constexpr int T = 16 * TB;
  __shared__ float4 sa[8][T];
  __shared__ float4 sb[8][T];
  __shared__ uint32_t red[8];
  const int t = blockIdx.z;
  // triangle index -> tile (bi, bj), bi <= bj
  const int tri = blockIdx.x;
  int bj = (int)((sqrtf(8.0f * (float)tri + 1.0f) - 1.0f) * 0.5f);
  while ((bj + 1) * (bj + 2) / 2 <= tri) bj++;
  while (bj * (bj + 1) / 2 > tri) bj--;
  const int bi = tri - bj * (bj + 1) / 2;
  const int i0 = bi * T, j0 = bj * T;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int32_t *c = cand + (int64_t)t * R;
  float acc[TB][TB];
#pragma unroll
  for (int a = 0; a < TB; a++)
#pragma unroll
    for (int b = 0; b < TB; b++) acc[a][b] = 0.0f;
  for (int ch = 0; ch < dp4; ch += 8) {
    const int nch = min(8, dp4 - ch);
    for (int e = threadIdx.x; e < T * 8; e += 256) {
      const int r = e % T, q = e / T;
      const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
      sa[q][r] = (q < nch && i0 + r < R) ? rows[(int64_t)c[i0 + r] * dp4 + ch + q] : zero;
      sb[q][r] = (q < nch && j0 + r < R) ? rows[(int64_t)c[j0 + r] * dp4 + ch + q] : zero;
    }
    __syncthreads();
    for (int q = 0; q < nch; q++) {
      float4 av[TB], bv[TB];
#pragma unroll
      for (int a = 0; a < TB; a++) av[a] = sa[q][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < TB; b++) bv[b] = sb[q][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < TB; a++)
#pragma unroll
        for (int b = 0; b < TB; b++) {
          float s = acc[a][b], u;
          u = __fsub_rn(av[a].x, bv[b].x); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].y, bv[b].y); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].z, bv[b].z); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].w, bv[b].w); s = __fmaf_rn(u, u, s);
          acc[a][b] = s;
        }
    }
    __syncthreads();
  }
  uint32_t sum = 0;
#pragma unroll
  for (int a = 0; a < TB; a++)
#pragma unroll
    for (int b = 0; b < TB; b++)
      if (i0 + ty + 16 * a < R && j0 + tx + 16 * b < R)
        sum += (uint32_t)(int32_t)sqrtf(acc[a][b]);
  // block reduce (wrapping unsigned add), one atomic per block
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < 8; w++) tot += red[w];
    atomicAdd(score + t, bi == bj ? tot : 2u * tot);
  }
}

// Picks the first trial whose score, compared as float against a running
// best starting at 0.0f, is larger (selectReps_max, knnjoin.cu:135-148) and
// gathers its rows.  Every block picks the trial (a few hundred scores at
// most) and copies a slice of the rows.
__global__ void rep_pick_kernel(const float4 *__restrict__ rows, int dp4,
                                const int32_t *__restrict__ cand, int R,
                                int trials, const uint32_t *__restrict__ score,
                                float4 *__restrict__ reps,
                                int32_t *__restrict__ rep_rows) {
  __shared__ int best_s;
  if (threadIdx.x == 0) {
    float best = 0.0f;
    int bt = 0;
    for (int t = 0; t < trials; t++) {
      float v = (float)(int32_t)score[t];
      if (best < v) {
        best = v;
        bt = t;
      }
    }
    best_s = bt;
  }
  __syncthreads();
  const int32_t *c = cand + (int64_t)best_s * R;
  const int64_t total = (int64_t)R * dp4;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / dp4), kk = (int)(e - (int64_t)i * dp4);
    const int32_t row = c[i];
    if (kk == 0 && rep_rows) rep_rows[i] = row;
    reps[e] = rows[(int64_t)row * dp4 + kk];
  }
}

// ---------------------------------------------------------------------------
// Nearest representative (findQCluster / findTCluster, knnjoin.cu:64-97):
// argmin over representatives of the FP32 distance, lowest representative
// index on ties.  The reference computes the distances as
// sqrt(|x|^2 + |r|^2 - 2 x.r) through cuBLAS (knnjoin.cu:270-284, 55-63);
// here they are computed directly, which cannot go negative.
// Representatives are staged through shared memory in tiles.
// ---------------------------------------------------------------------------
template <int DP4>
__global__ void __launch_bounds__(256)
    assign_kernel(const float4 *__restrict__ rows, int64_t n,
                  const float4 *__restrict__ reps, int R,
                  int32_t *__restrict__ cl, float *__restrict__ dr) {
  constexpr int TILE = (DP4 <= 2) ? 1024 : (DP4 <= 4 ? 512 : 256);
  __shared__ float4 srep[TILE * DP4];
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float4 p[DP4];
#pragma unroll
  for (int c = 0; c < DP4; c++)
    p[c] = i < n ? rows[i * DP4 + c] : make_float4(0.f, 0.f, 0.f, 0.f);
  // bi starts at 0 so that a point with a NaN coordinate (no comparison
  // succeeds) still lands in a valid cluster.
  float best = __int_as_float(0x7f7fffff);  // FLT_MAX
  int bi = 0;
  for (int base = 0; base < R; base += TILE) {
    int cnt = min(TILE, R - base);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * DP4; t += blockDim.x)
      srep[t] = reps[(int64_t)base * DP4 + t];
    __syncthreads();
    for (int j = 0; j < cnt; j++) {
      float v = dist2_rows<DP4>(p, srep + j * DP4);
      if (v < best) {
        best = v;
        bi = base + j;
      }
    }
  }
  if (i < n) {
    cl[i] = bi;
    dr[i] = sqrtf(best);
  }
}

// Runtime-width variant for rows wider than 32 floats: the point row is read
// through the read-only cache for every representative.
__global__ void __launch_bounds__(256)
    assign_kernel_rt(const float4 *__restrict__ rows, int64_t n, int dp4,
                     const float4 *__restrict__ reps, int R,
                     int32_t *__restrict__ cl, float *__restrict__ dr) {
  extern __shared__ float4 srep_rt[];
  const int TILE = 8192 / dp4 > 0 ? 8192 / dp4 : 1;  // 128 KB of float4
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const float4 *p = rows + (i < n ? i : 0) * dp4;
  float best = __int_as_float(0x7f7fffff);
  int bi = 0;
  for (int base = 0; base < R; base += TILE) {
    int cnt = min(TILE, R - base);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * dp4; t += blockDim.x)
      srep_rt[t] = reps[(int64_t)base * dp4 + t];
    __syncthreads();
    for (int j = 0; j < cnt; j++) {
      float v = dist2_rows_rt(p, srep_rt + j * dp4, dp4);
      if (v < best) {
        best = v;
        bi = base + j;
      }
    }
  }
  if (i < n) {
    cl[i] = bi;
    dr[i] = sqrtf(best);
  }
}

// Lloyd step: every representative moves to the centroid of its members.
// One block per cluster; members are read in cluster order (perm) and summed
// with a fixed assignment of members to threads and a fixed tree, so the
// result does not depend on scheduling.  Empty clusters keep their
// representative.  (Representative refinement is not in the reference, which
// keeps the best of its random draws, knnjoin.cu:125-154.)
__global__ void __launch_bounds__(256)
    centroid_kernel(const float4 *__restrict__ rows, int dp4, const int32_t *__restrict__ perm,
                    const int32_t *__restrict__ off, float4 *__restrict__ reps) {
  // G = pow2 >= dp4 lanes read one member row (one float4 each, coalesced);
  // 256 / G groups take every (256/G)-th member; the groups' partial sums are
  // added in group order, so the result does not depend on scheduling.
  __shared__ float4 red[256];
  const int c = blockIdx.x, tid = threadIdx.x;
  const int a = off[c], b = off[c + 1];
  if (b == a) return;
  int G = 1;
  while (G < dp4 && G < 256) G <<= 1;
  const int groups = 256 / G, g = tid / G, col = tid % G;
  for (int c0 = 0; c0 < dp4; c0 += G) {
    const int ch = c0 + col;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ch < dp4 && g < groups)
      for (int p = a + g; p < b; p += groups) {
        const float4 v = rows[(int64_t)perm[p] * dp4 + ch];
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += v.w;
      }
    red[tid] = acc;
    __syncthreads();
    if (tid < G && c0 + tid < dp4) {
      float4 t = red[tid];
      for (int h = 1; h < groups; h++) {
        const float4 v = red[h * G + tid];
        t.x += v.x;
        t.y += v.y;
        t.z += v.z;
        t.w += v.w;
      }
      const float inv = 1.0f / (float)(b - a);
      reps[(int64_t)c * dp4 + c0 + tid] = make_float4(t.x * inv, t.y * inv, t.z * inv, t.w * inv);
    }
    __syncthreads();
  }
}

int launch_centroids(const float4 *rows, int dp4, const int32_t *perm, const int32_t *off, int R,
                     float4 *reps, cudaStream_t s) {
  centroid_kernel<<<R, 256, 0, s>>>(rows, dp4, perm, off, reps);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

// ---------------------------------------------------------------------------
// Cluster split (refinement steps only; the reference has no counterpart).
// A random draw leaves some dense regions without a representative; their
// points join a distant cluster whose radius then spans both regions, and
// such clusters defeat the triangle-inequality bounds.  Each refinement step
// pairs the smallest clusters (donors) with the widest ones (receivers) and
// moves each donor's representative onto its receiver's farthest member, so
// the next assignment splits the receiver.  A pair moves only when the
// receiver's radius is more than twice the median radius and the donor holds
// fewer points than the median cluster.  Deterministic: both orders break
// ties by cluster id.  One block; R <= 8192.
// dynamic shared memory: 2 * pow2(R) keys
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
    split_clusters_kernel(const float4 *__restrict__ rows, int dp4,
                          const int32_t *__restrict__ perm, const int32_t *__restrict__ off,
                          const uint64_t *__restrict__ skeys, int R, int rp2, int max_moves,
                          float4 *__restrict__ reps) {
  extern __shared__ uint64_t sk[];
  uint64_t *by_size = sk, *by_radius = sk + rp2;
  const int tid = threadIdx.x;
  for (int c = tid; c < rp2; c += blockDim.x) {
    uint64_t ks = kKeyMax, kr = kKeyMax;
    if (c < R) {
      const int a = off[c], b = off[c + 1];
      const float rad = b > a ? __uint_as_float((uint32_t)skeys[b - 1]) : 0.0f;
      ks = ((uint64_t)(uint32_t)(b - a) << 32) | (uint32_t)c;
      kr = ((uint64_t)(~__float_as_uint(rad)) << 32) | (uint32_t)c;  // widest first
    }
    by_size[c] = ks;
    by_radius[c] = kr;
  }
  __syncthreads();
  for (int size = 2; size <= rp2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = tid; t < rp2 / 2; t += blockDim.x) {
        const int i = 2 * t - (t & (stride - 1)), j = i + stride;
        const bool up = (i & size) == 0;
        uint64_t x = by_size[i], y = by_size[j];
        if ((x > y) == up) {
          by_size[i] = y;
          by_size[j] = x;
        }
        x = by_radius[i];
        y = by_radius[j];
        if ((x > y) == up) {
          by_radius[i] = y;
          by_radius[j] = x;
        }
      }
      __syncthreads();
    }
  }
  const float med_rad = __uint_as_float(~(uint32_t)(by_radius[R / 2] >> 32));
  const uint32_t med_size = (uint32_t)(by_size[R / 2] >> 32);
  for (int i = tid; i < max_moves; i += blockDim.x) {
    const int recv = (int)(uint32_t)by_radius[i];
    const int donor = (int)(uint32_t)by_size[i];
    const float rad = __uint_as_float(~(uint32_t)(by_radius[i] >> 32));
    const uint32_t dsize = (uint32_t)(by_size[i] >> 32);
    if (recv == donor || !(rad > 2.0f * med_rad) || dsize >= med_size) continue;
    const int far = perm[off[recv + 1] - 1];
    for (int ch = 0; ch < dp4; ch++) reps[(int64_t)donor * dp4 + ch] = rows[(int64_t)far * dp4 + ch];
  }
}

int launch_split_clusters(const float4 *rows, int dp4, const int32_t *perm, const int32_t *off,
                          const uint64_t *skeys, int R, float4 *reps, cudaStream_t s) {
  if (R < 4) return KNN_OK;
  int rp2 = 1;
  while (rp2 < R) rp2 <<= 1;
  const size_t smem = 2 * (size_t)rp2 * sizeof(uint64_t);
  if (smem > 48 * 1024)
    KNN_CUDA_TRY(cudaFuncSetAttribute(split_clusters_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  split_clusters_kernel<<<1, 1024, smem, s>>>(rows, dp4, perm, off, skeys, R, rp2,
                                              std::max(1, R / 16), reps);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

// Sort keys (cluster << 32 | distance bits) and identity values.
__global__ void cluster_keys_kernel(const int32_t *__restrict__ cl,
                                    const float *__restrict__ dr, int64_t n,
                                    uint64_t *__restrict__ keys,
                                    int32_t *__restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    keys[i] = ((uint64_t)(uint32_t)cl[i] << 32) | __float_as_uint(dr[i]);
    vals[i] = (int32_t)i;
  }
}

// Cluster-contiguous layout: row p of the sorted set is input row perm[p];
// its distance to the representative is the low word of its key.
// (fillTMembers + host sort, knnjoin.cu:106-113, 382-399, without the
// per-cluster device<->host round trips.)  With idx_in_row the last pad float
// of every row carries the original row index, so the scan gets coordinates
// and index from one load.
__global__ void cluster_layout_kernel(const uint64_t *__restrict__ skeys,
                                      const int32_t *__restrict__ perm,
                                      int64_t n, const float4 *__restrict__ rows,
                                      int dp4, bool idx_in_row,
                                      float4 *__restrict__ srows,
                                      float *__restrict__ sdist,
                                      int32_t *__restrict__ sidx) {
  int64_t total = n * dp4;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t p = t / dp4;
    int c = (int)(t - p * dp4);
    int32_t src = perm[p];
    float4 v = rows[(int64_t)src * dp4 + c];
    if (idx_in_row && c == dp4 - 1) v.w = __int_as_float(src);
    srows[t] = v;
    if (c == 0) {
      if (sdist) sdist[p] = __uint_as_float((uint32_t)(skeys[p] & 0xffffffffu));
      if (sidx) sidx[p] = src;
    }
  }
}

// Offsets of every cluster in the sorted order (off[R] = n) from the sorted
// keys, plus min / max member distance (the reference never fills the
// reference-cluster radius: knnjoin.cu:391, defect B1).
__global__ void cluster_bounds_kernel(const uint64_t *__restrict__ skeys,
                                      int64_t n, int R,
                                      int32_t *__restrict__ off) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(skeys[p] >> 32);
    int prev = p == 0 ? -1 : (int)(skeys[p - 1] >> 32);
    for (int x = prev + 1; x <= c; x++) off[x] = (int32_t)p;
    if (p == n - 1)
      for (int x = c + 1; x <= R; x++) off[x] = (int32_t)n;
  }
}

__global__ void cluster_minmax_kernel(const int32_t *__restrict__ off,
                                      const float *__restrict__ sdist, int R,
                                      float *__restrict__ cmin,
                                      float *__restrict__ cmax) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < R) {
    int a = off[c], b = off[c + 1];
    cmin[c] = b > a ? sdist[a] : 0.0f;
    cmax[c] = b > a ? sdist[b - 1] : 0.0f;
  }
}

// Same for clusters of the query set when only the maximum is needed
// (maxquery, knnjoin.cu:78).
__global__ void cluster_max_from_keys_kernel(const uint64_t *__restrict__ skeys,
                                             const int32_t *__restrict__ off,
                                             int R, float *__restrict__ cmax) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < R) {
    int a = off[c], b = off[c + 1];
    cmax[c] = b > a ? __uint_as_float((uint32_t)(skeys[b - 1] & 0xffffffffu)) : 0.0f;
  }
}

// Cluster id of every query slot in the sorted query order.
__global__ void slot_cluster_kernel(const uint64_t *__restrict__ skeys,
                                    int64_t m, int32_t *__restrict__ slot_cl) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m;
       p += (int64_t)gridDim.x * blockDim.x)
    slot_cl[p] = (int32_t)(skeys[p] >> 32);
}

// d(Rq_a, Rs_b) for all pairs (the reference recomputes these inside
// RepsUpperBound and FilterReps: knnjoin.cu:468, 513).  Tiled like the
// spread score: a block owns 64 x 64 pairs, rows staged through shared memory
// 32 floats at a time, 16 pairs per thread, each summed in dimension order
// with fma (the same value as the one-pair distance).
// grid: (ceil(Rq / 64), ceil(Rs / 64)), 256 threads
__global__ void __launch_bounds__(256)
    rep_dist_kernel(const float4 *__restrict__ qreps, int Rq, const float4 *__restrict__ sreps,
                    int Rs, int dp4, float *__restrict__ drr) {
  __shared__ float4 sa[8][64];
  __shared__ float4 sb[8][64];
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0f;
  for (int ch = 0; ch < dp4; ch += 8) {
    const int nch = min(8, dp4 - ch);
    for (int e = threadIdx.x; e < 64 * 8; e += 256) {
      const int r = e & 63, q = e >> 6;
      const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
      sa[q][r] = (q < nch && i0 + r < Rq) ? qreps[(int64_t)(i0 + r) * dp4 + ch + q] : zero;
      sb[q][r] = (q < nch && j0 + r < Rs) ? sreps[(int64_t)(j0 + r) * dp4 + ch + q] : zero;
    }
    __syncthreads();
    for (int q = 0; q < nch; q++) {
      float4 av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; a++) av[a] = sa[q][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; b++) bv[b] = sb[q][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          float s = acc[a][b], u;
          u = __fsub_rn(av[a].x, bv[b].x); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].y, bv[b].y); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].z, bv[b].z); s = __fmaf_rn(u, u, s);
          u = __fsub_rn(av[a].w, bv[b].w); s = __fmaf_rn(u, u, s);
          acc[a][b] = s;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < Rq && j < Rs) drr[(int64_t)i * Rs + j] = sqrtf(acc[a][b]);
    }
}

// dynamic shared memory: RsPow2 * 8 bytes (sort keys).
__global__ void __launch_bounds__(512)
    bounds_filter_kernel(const float *__restrict__ drr, int Rq, int Rs,
                         const float *__restrict__ qrad,
                         const int32_t *__restrict__ qoff,
                         const int32_t *__restrict__ soff,
                         const float *__restrict__ sdist,
                         const float *__restrict__ scmax, int k, int d,
                         int rs_pow2, float *__restrict__ theta0,
                         int32_t *__restrict__ rlist,
                         int32_t *__restrict__ rlen, float2 *__restrict__ clb) {
  extern __shared__ uint64_t skey[];
  const int qc = blockIdx.x;
  if (qoff[qc + 1] == qoff[qc]) {  // empty query cluster
    if (threadIdx.x == 0) {
      theta0[qc] = 0.0f;
      rlen[qc] = 0;
    }
    return;
  }
  bounds_filter_block(drr + (int64_t)qc * Rs, Rs, soff, sdist, scmax, qrad[qc], k, d, rs_pow2,
                      0, skey, theta0 + qc, rlist + (int64_t)qc * Rs, rlen + qc,
                      clb ? clb + (int64_t)qc * ((Rs + 31) / 32) : nullptr);
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
static int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  int64_t cap = 148LL * 32;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

// Exactness of FP32 distances: raises *inexact unless every value of x is an
// integer of magnitude at most `bound`.  With bound = sqrt(2^24 / d) / 2 every
// coordinate difference, square and partial sum of a squared distance is an
// integer below 2^24, so the FP32 squared distance is exact, equal to the FP64
// one, and the two rank every pair alike (the k-th boundary needs no FP64
// re-check).  The reference's sample data (integer RGB values) is of this
// kind.
__global__ void exact_check_kernel(const float *__restrict__ x, int64_t count, float bound,
                                   int *inexact) {
  bool bad = false;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[t];
    bad |= !(v == rintf(v) && fabsf(v) <= bound);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(inexact, 1);
}

// Estimated search work of every query cluster, to balance a partition of
// the query clusters across devices (the reference runs its whole search on
// one GPU, src/knnjoin.cu:1103-1129): the cluster's query count times the
// summed sizes of the bands it can scan, each taken for the cluster as a
// whole (members s of a surviving reference cluster Rs with
// |d(Rq,Rs) - d(s,Rs)| <= rq + theta0), plus one per query.  One warp per
// query cluster.
__global__ void cluster_work_kernel(const float *__restrict__ drr, int Rq, int Rs,
                                    const float *__restrict__ qrad,
                                    const float *__restrict__ theta0,
                                    const int32_t *__restrict__ qoff,
                                    const int32_t *__restrict__ rlist,
                                    const int32_t *__restrict__ rlen,
                                    const int32_t *__restrict__ soff,
                                    const float *__restrict__ sdist, long long *__restrict__ work) {
  const int lane = threadIdx.x & 31;
  const int qc = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (qc >= Rq) return;
  const float w = qrad[qc] + theta0[qc];
  long long band = 0;
  for (int j = lane; j < rlen[qc]; j += 32) {
    const int rs = rlist[(int64_t)qc * Rs + j];
    const float D = drr[(int64_t)qc * Rs + rs];
    const int a = soff[rs], n = soff[rs + 1] - a;
    int lo = 0, hi = n;  // first member >= D - w
    while (lo < hi) {
      const int md = (lo + hi) >> 1;
      if (sdist[a + md] < D - w) lo = md + 1;
      else hi = md;
    }
    int l2 = lo, h2 = n;  // first member > D + w
    while (l2 < h2) {
      const int md = (l2 + h2) >> 1;
      if (sdist[a + md] <= D + w) l2 = md + 1;
      else h2 = md;
    }
    band += l2 - lo;
  }
  for (int o = 16; o > 0; o >>= 1) band += __shfl_xor_sync(0xffffffffu, band, o);
  if (lane == 0) {
    const long long nq = qoff[qc + 1] - qoff[qc];
    work[qc] = nq * (band + 1);
  }
}

int launch_cluster_work(const float *drr, int Rq, int Rs, const float *qrad, const float *theta0,
                        const int32_t *qoff, const int32_t *rlist, const int32_t *rlen,
                        const int32_t *soff, const float *sdist, long long *work,
                        cudaStream_t s) {
  if (Rq == 0) return KNN_OK;
  cluster_work_kernel<<<(Rq + 7) / 8, 256, 0, s>>>(drr, Rq, Rs, qrad, theta0, qoff, rlist, rlen,
                                                 soff, sdist, work);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_exact_check(const float *x, int64_t count, int d, int *inexact, cudaStream_t s) {
  if (count == 0) return KNN_OK;
  const float bound = floorf(sqrtf(16777216.0f / (float)d) * 0.5f);
  exact_check_kernel<<<grid_for(count, 256), 256, 0, s>>>(x, count, bound, inexact);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_pack_rows(const float *src, int64_t n, int d, int dp4, float4 *dst,
                     cudaStream_t s) {
  if (n == 0) return KNN_OK;
  pack_rows_kernel<<<grid_for(n * dp4, 256), 256, 0, s>>>(src, n, d, dp4, dst);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_rep_select(const float4 *rows, int dp4, const int32_t *cand_dev,
                      int R, int trials, uint32_t *score_dev, float4 *reps,
                      int32_t *rep_rows, cudaStream_t s) {
  KNN_CUDA_TRY(cudaMemsetAsync(score_dev, 0, sizeof(uint32_t) * trials, s));
  // a single draw needs no score (the pick keeps trial 0 either way)
  if (trials > 1) {
    // 4 x 4 pairs per thread: 8 x 8 (fewer shared-memory loads per fma) took
    // about 160 registers and measured slower on 8,192 representatives
    const int nb = (R + 63) / 64;
    dim3 grid((unsigned)(nb * (nb + 1) / 2), 1, trials);
    rep_score_kernel<4><<<grid, 256, 0, s>>>(rows, dp4, cand_dev, R, score_dev);
    KNN_LAUNCH_CHECK();
  }
  const int64_t words = (int64_t)R * dp4;
  const int pick_blocks = (int)std::min<int64_t>(1024, std::max<int64_t>(1, (words + 255) / 256));
  rep_pick_kernel<<<pick_blocks, 256, 0, s>>>(rows, dp4, cand_dev, R, trials, score_dev, reps,
                                              rep_rows);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_assign(const float4 *rows, int64_t n, int dp4, const float4 *reps,
                  int R, int32_t *cl, float *dr, cudaStream_t s) {
  if (n == 0) return KNN_OK;
  int blocks = (int)((n + 255) / 256);
  switch (dp4) {
#define KNN_ASSIGN_CASE(D)                                                   \
  case D:                                                                    \
    assign_kernel<D><<<blocks, 256, 0, s>>>(rows, n, reps, R, cl, dr);       \
    break;
    KNN_ASSIGN_CASE(1)
    KNN_ASSIGN_CASE(2)
    KNN_ASSIGN_CASE(3)
    KNN_ASSIGN_CASE(4)
    KNN_ASSIGN_CASE(5)
    KNN_ASSIGN_CASE(6)
    KNN_ASSIGN_CASE(7)
    KNN_ASSIGN_CASE(8)
#undef KNN_ASSIGN_CASE
    default: {
      int tile = 8192 / dp4 > 0 ? 8192 / dp4 : 1;
      size_t smem = (size_t)tile * dp4 * sizeof(float4);
      if (smem > 48 * 1024)
        KNN_CUDA_TRY(cudaFuncSetAttribute(
            assign_kernel_rt, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)smem));
      assign_kernel_rt<<<blocks, 256, smem, s>>>(rows, n, dp4, reps, R, cl, dr);
    }
  }
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

size_t cluster_sort_temp_bytes(int64_t n, int R) {
  size_t bytes = 0;
  int end_bit = 32;
  while ((1LL << (end_bit - 32)) < (int64_t)R) end_bit++;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t *)nullptr,
                                  (uint64_t *)nullptr, (const int32_t *)nullptr,
                                  (int32_t *)nullptr, (int)n, 0, end_bit);
  return bytes;
}

// Query slots grouped by row chunk: chunk c holds the slots of query rows
// [c * chunk_rows, (c + 1) * chunk_rows), in slot (query-cluster) order -- a
// stable radix sort of the slots by chunk id.
__global__ void chunk_keys_kernel(const int32_t *__restrict__ qorder, int64_t m, int first,
                                  int chunk_rows, uint32_t *__restrict__ keys,
                                  int32_t *__restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t row = qorder[i];
    keys[i] = first > 0 ? (row < first ? 0u : 1u + (uint32_t)((row - first) / chunk_rows))
                        : (uint32_t)(row / chunk_rows);
    vals[i] = (int32_t)i;
  }
}

static int chunk_bits(int nchunks) {
  int b = 1;
  while ((1 << b) < nchunks) b++;
  return b;
}

size_t chunk_slots_temp_bytes(int64_t m, int nchunks) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint32_t *)nullptr,
                                  (uint32_t *)nullptr, (const int32_t *)nullptr,
                                  (int32_t *)nullptr, (int)m, 0, chunk_bits(nchunks));
  return bytes;
}

int launch_chunk_slots(const int32_t *qorder, int64_t m, int first, int chunk_rows, int nchunks,
                       uint32_t *keys, uint32_t *keys_out, int32_t *vals, int32_t *slots,
                       void *temp, size_t temp_bytes, cudaStream_t s) {
  chunk_keys_kernel<<<grid_for(m, 256), 256, 0, s>>>(qorder, m, first, chunk_rows, keys, vals);
  KNN_LAUNCH_CHECK();
  KNN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_out, vals, slots,
                                               (int)m, 0, chunk_bits(nchunks), s));
  ++launch_counter();
  return KNN_OK;
}

int launch_cluster_sort(const int32_t *cl, const float *dr, int64_t n, int R,
                        uint64_t *keys, int32_t *vals, uint64_t *skeys,
                        int32_t *perm, void *temp, size_t temp_bytes,
                        cudaStream_t s) {
  if (n == 0) return KNN_OK;
  cluster_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(cl, dr, n, keys, vals);
  KNN_LAUNCH_CHECK();
  int end_bit = 32;
  while ((1LL << (end_bit - 32)) < (int64_t)R) end_bit++;
  KNN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, skeys,
                                               vals, perm, (int)n, 0, end_bit, s));
  ++launch_counter();
  return KNN_OK;
}

int launch_cluster_layout(const uint64_t *skeys, const int32_t *perm, int64_t n,
                          const float4 *rows, int dp4, bool idx_in_row,
                          float4 *srows, float *sdist, int32_t *sidx,
                          cudaStream_t s) {
  if (n == 0) return KNN_OK;
  cluster_layout_kernel<<<grid_for(n * dp4, 256), 256, 0, s>>>(
      skeys, perm, n, rows, dp4, idx_in_row, srows, sdist, sidx);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_cluster_offsets(const uint64_t *skeys, int64_t n, int R, int32_t *off,
                           cudaStream_t s) {
  if (n == 0) {
    KNN_CUDA_TRY(cudaMemsetAsync(off, 0, sizeof(int32_t) * (R + 1), s));
    return KNN_OK;
  }
  cluster_bounds_kernel<<<grid_for(n, 256), 256, 0, s>>>(skeys, n, R, off);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_cluster_minmax(const int32_t *off, const float *sdist, int R,
                          float *cmin, float *cmax, cudaStream_t s) {
  cluster_minmax_kernel<<<(R + 255) / 256, 256, 0, s>>>(off, sdist, R, cmin, cmax);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_query_clusters(const uint64_t *skeys, const int32_t *off, int64_t m,
                          int R, float *qrad, int32_t *slot_cl, cudaStream_t s) {
  cluster_max_from_keys_kernel<<<(R + 255) / 256, 256, 0, s>>>(skeys, off, R, qrad);
  KNN_LAUNCH_CHECK();
  if (m > 0) {
    slot_cluster_kernel<<<grid_for(m, 256), 256, 0, s>>>(skeys, m, slot_cl);
    KNN_LAUNCH_CHECK();
  }
  return KNN_OK;
}

int launch_rep_dist(const float4 *qreps, int Rq, const float4 *sreps, int Rs,
                    int dp4, float *drr, cudaStream_t s) {
  if ((int64_t)Rq * Rs == 0) return KNN_OK;
  rep_dist_kernel<<<dim3((Rq + 63) / 64, (Rs + 63) / 64), 256, 0, s>>>(qreps, Rq, sreps, Rs,
                                                                      dp4, drr);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

int launch_bounds_filter(const float *drr, int Rq, int Rs, const float *qrad,
                         const int32_t *qoff, const int32_t *soff,
                         const float *sdist, const float *scmax, int k, int d,
                         float *theta0, int32_t *rlist, int32_t *rlen,
                         float2 *clb, cudaStream_t s) {
  int p2 = 1;
  while (p2 < Rs) p2 <<= 1;
  size_t smem = (size_t)p2 * sizeof(uint64_t);
  if (smem > 48 * 1024)
    KNN_CUDA_TRY(cudaFuncSetAttribute(bounds_filter_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  bounds_filter_kernel<<<Rq, 512, smem, s>>>(drr, Rq, Rs, qrad, qoff, soff, sdist,
                                             scmax, k, d, p2, theta0, rlist, rlen, clb);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

}  // namespace knnsweet
