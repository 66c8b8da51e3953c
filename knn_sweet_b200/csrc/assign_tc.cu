// assign_tc.cu -- nearest representative on the tensor cores (tcgen05).
//
// For rows wide enough to be a dense contraction (d >= 16) the assignment of
// every point to its nearest representative (findQCluster / findTCluster,
// src/knnjoin.cu:64-97, over the cuBLAS distance matrix of knnjoin.cu:270-342)
// is an n x R x d GEMM with an arg-max epilogue:
//     argmax_j  p . r_j - |r_j|^2 / 2
// computed from BF16-rounded points and representatives with FP32 accumulation
// in TMEM; the norm term rides in three extra contraction columns.  The
// choice only has to be approximately nearest: the pruning bounds need the
// exact distance to whichever representative is chosen, and that distance is
// recomputed in FP32 at the end of the kernel.
//
// One CTA (8 epilogue warps + 1 producer warp) owns 128 points: all warps
// convert them to BF16 into shared memory in the core-matrix layout of
// tc_common.cuh while the first two tiles of TN = 128 representatives
// (pre-converted once, contiguous) arrive by bulk asynchronous copy; the
// producer issues KD/16 MMAs (M = 128, N = TN, K = 16) per tile into one of
// two TMEM accumulators and commits to an mbarrier; the epilogue warps read
// the rows back (tcgen05.ld 32x32b) and keep a running arg-max per row while
// the next tile's MMA runs.  Every wait is bounded; on timeout the CTA flags
// the error, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_common.cuh"

namespace knnsweet {

namespace {
constexpr int kTileM = 128;  // points per CTA (TMEM lanes)
constexpr int kTileN = 256;  // representatives per MMA (TMEM columns)
}  // namespace

// Representatives -> BF16 tiles of kTileN rows in the core-matrix layout.
// Columns d, d+1 and d+2 carry the squared norm of the BF16-rounded row,
// split into three BF16 parts whose sum is the FP32 norm (8 significant bits
// each); the points carry -0.5 there, so the MMA yields p.r - |r|^2 / 2 and
// the nearest representative is its arg-max.  Padding rows carry the largest
// finite BF16 value as the norm: they never win.
__global__ void reps_to_bf16_tiles_kernel(const float4 *__restrict__ reps, int R, int dp4,
                                          int d, int KD, int Rpad,
                                          __nv_bfloat16 *__restrict__ tiles) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Rpad) return;
  unsigned char *tile = reinterpret_cast<unsigned char *>(tiles) +
                        (size_t)(r / kTileN) * tc::tile_bytes(kTileN, KD);
  const int rr = r % kTileN;
  auto coord = [&](int k) -> float {
    const float4 c = reps[(size_t)r * dp4 + (k >> 2)];
    return (k & 3) == 0 ? c.x : (k & 3) == 1 ? c.y : (k & 3) == 2 ? c.z : c.w;
  };
  __nv_bfloat16 part[3];
  if (r < R) {
    float nrm = 0.0f;
    for (int k = 0; k < d; k++) {
      const float xr = __bfloat162float(__float2bfloat16_rn(coord(k)));
      nrm = __fmaf_rn(xr, xr, nrm);
    }
    // each remainder is exact in FP32: the part is the remainder rounded
#pragma unroll
    for (int t = 0; t < 3; t++) {
      part[t] = __float2bfloat16_rn(nrm);
      nrm -= __bfloat162float(part[t]);
    }
  } else {
    part[0] = __ushort_as_bfloat16(0x7f7f);
    part[1] = part[2] = __float2bfloat16_rn(0.0f);
  }
  for (int k0 = 0; k0 < KD; k0 += 8) {
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int k = k0 + e;
      v[e] = k >= d && k < d + 3 ? part[k - d]
             : (r < R && k < d)  ? __float2bfloat16_rn(coord(k))
                                 : __float2bfloat16_rn(0.0f);
    }
    *reinterpret_cast<uint4 *>(tile + tc::tile_offset(rr, k0, KD)) =
        *reinterpret_cast<const uint4 *>(v);
  }
}

// Warp-specialised arg-max: warps 0-7 (the epilogue) own 128 points, warp 8
// (the producer) streams the representative tiles (pre-converted,
// contiguous) through two shared-memory buffers by 1-D bulk asynchronous
// copies that complete on an mbarrier transaction count, and issues the MMAs
// into two TMEM accumulators of TN columns.  The accumulator holds
// p.r - |r|^2 / 2 (norm columns folded into the contraction), so the
// epilogue is a bare arg-max.  Handshakes, all mbarriers, no CTA barrier in
// the loop:
//   full[b]   copy of the tile in buffer b landed        (producer waits)
//   done[b]   MMA into accumulator b finished            (both wait)
//   empty[b]  8 epilogue warps finished reading b        (producer waits)
// Warps w and w+4 read the same 32 TMEM lanes (rows) and split the TN
// columns; each thread keeps four independent running maxima (column c goes
// to chain c % 4), merged by (value, index) at the end so ties still go to
// the lowest index.  Any wait that gives up raises a shared abort flag that
// the other warps check before their next wait.
// dynamic shared memory: A tile, 2 B tiles, 6 mbarriers, TMEM slot, abort
// flag, 128 (value, index) pairs
// epilogue warps split the TN columns kEsplit ways (4 measured no faster)
constexpr int kEsplit = 2;
constexpr int kAssignThreads = 128 * kEsplit + 32;
// Representative tile width (MMA N) and the number of shared-memory tile
// buffers the producer keeps in flight: a buffer is refilled with tile
// j + kStages once MMA j has read it.
#ifndef KNN_ASSIGN_TN
#define KNN_ASSIGN_TN 128
#endif
#ifndef KNN_ASSIGN_STAGES
#define KNN_ASSIGN_STAGES 2
#endif
constexpr int kStages = KNN_ASSIGN_STAGES;

__global__ void __launch_bounds__(kAssignThreads, 1)
    assign_tc_kernel(const float4 *__restrict__ rows, int64_t n, int dp4, int d, int KD, int TN,
                     const __nv_bfloat16 *__restrict__ rep_tiles, int ntiles,
                     const float4 *__restrict__ reps, int R, int32_t *__restrict__ cl,
                     float *__restrict__ dr, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const size_t a_bytes = tc::tile_bytes(kTileM, KD), b_bytes = tc::tile_bytes(TN, KD);
  unsigned char *sa = smem;
  unsigned char *sb0 = sa + a_bytes;
  auto sb = [&](int b) { return sb0 + (size_t)b * b_bytes; };
  uint64_t *full = reinterpret_cast<uint64_t *>(sb0 + (size_t)kStages * b_bytes);
  uint64_t *done = full + kStages;
  uint64_t *empty = done + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(empty + 2);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  float *pv = reinterpret_cast<float *>(tmem_slot + 4);  // kEsplit x 128 partial maxima
  int *pi = reinterpret_cast<int *>(pv + kEsplit * kTileM);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t row0 = (int64_t)blockIdx.x * kTileM;
  const uint32_t ncols = 2u * (uint32_t)TN;  // 256 or 512, a power of two
  const unsigned char *tiles_g = reinterpret_cast<const unsigned char *>(rep_tiles);

  if (warp == 0) tc::tmem_alloc(tmem_slot, ncols);
  if (tid == 0) {
    for (int i = 0; i < kStages; i++) tc::mbar_init(full + i, 1);
    for (int i = 0; i < 2; i++) {
      tc::mbar_init(done + i, 1);
      tc::mbar_init(empty + i, 4 * kEsplit);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool producer = warp == 4 * kEsplit && lane == 0;
  // the first kStages representative tiles in flight while the points are
  // staged
  if (producer)
    for (int j = 0; j < kStages && j < ntiles; j++) {
      tc::mbar_arrive_expect_tx(full + j, (uint32_t)b_bytes);
      tc::bulk_copy_g2s(sb(j), tiles_g + (size_t)j * b_bytes, (uint32_t)b_bytes, full + j);
    }
  // points -> BF16 core-matrix tile
  for (int t = tid; t < kTileM * (KD / 8); t += blockDim.x) {
    const int r = t / (KD / 8), k0 = (t % (KD / 8)) * 8;
    const int64_t gr = row0 + r;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int k = k0 + e;
      float x = 0.0f;
      if (gr < n && k < d) {
        const float4 c = rows[gr * dp4 + (k >> 2)];
        x = (k & 3) == 0 ? c.x : (k & 3) == 1 ? c.y : (k & 3) == 2 ? c.z : c.w;
      } else if (gr < n && k < d + 3) {
        x = -0.5f;  // times the representative's norm columns
      }
      v[e] = __float2bfloat16_rn(x);
    }
    *reinterpret_cast<uint4 *>(sa + tc::tile_offset(r, k0, KD)) =
        *reinterpret_cast<const uint4 *>(v);
  }
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  float bv = __int_as_float(0xff800000);
  int bi = 0;
  if (warp == 4 * kEsplit) {
    if (producer) {
      const uint32_t idesc = tc::make_idesc_bf16(kTileM, TN);
      const uint32_t a_base = tc::smem_u32(sa);
      const uint32_t sbo = (uint32_t)KD * 16;
      int copies = ntiles < kStages ? ntiles : kStages, mmas = 0;
      // MMA of tile j (buffer j % kStages) into accumulator j & 1, once its
      // copy landed and the epilogue released the accumulator (tile j - 2)
      auto issue = [&](int j) -> bool {
        const int b = j & 1, bb = j % kStages;
        if (j >= 2 && !tc::mbar_wait(empty + b, (uint32_t)(((j - 2) >> 1) & 1))) return false;
        if (!tc::mbar_wait(full + bb, (uint32_t)((j / kStages) & 1))) return false;
        tc::fence_after_sync();
        const uint32_t b_base = tc::smem_u32(sb(bb));
        for (int st = 0; st < KD / 16; st++) {
          const uint64_t ad = tc::make_desc(a_base + 256u * st, 128u, sbo);
          const uint64_t bd = tc::make_desc(b_base + 256u * st, 128u, sbo);
          tc::mma_bf16(tmem + (uint32_t)(b * TN), ad, bd, idesc, st > 0);
        }
        tc::mma_commit(done + b);
        mmas = j + 1;
        return true;
      };
      bool ok = ntiles == 0 || issue(0);
      for (int j = 0; ok && j < ntiles; j++) {
        if (*abort_flag) { ok = false; break; }
        // queue MMA j + 1 behind MMA j, then refill MMA j's buffer with
        // tile j + kStages once MMA j has read it
        if (j + 1 < ntiles && !issue(j + 1)) { ok = false; break; }
        if (j + kStages < ntiles) {
          const int bb = j % kStages;
          if (!tc::mbar_wait(done + (j & 1), (uint32_t)((j >> 1) & 1))) { ok = false; break; }
          tc::mbar_arrive_expect_tx(full + bb, (uint32_t)b_bytes);
          tc::bulk_copy_g2s(sb(bb), tiles_g + (size_t)(j + kStages) * b_bytes,
                            (uint32_t)b_bytes, full + bb);
          copies = j + kStages + 1;
        }
      }
      if (!ok) {
        *abort_flag = 1;
        // let the copies and MMAs already issued finish before the CTA's
        // shared memory and TMEM go away (bounded waits)
        for (int j = mmas; j < copies; j++)
          tc::mbar_wait(full + j % kStages, (uint32_t)((j / kStages) & 1));
        if (mmas > 0) tc::mbar_wait(done + ((mmas - 1) & 1), (uint32_t)(((mmas - 1) >> 1) & 1));
      }
    }
  } else {
    const int quad = warp & 3, part = warp >> 2;
    const int cbeg = part * (TN / kEsplit);
    float best[4];
    int bidx[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      best[c] = __int_as_float(0xff800000);
      bidx[c] = 0;
    }
    for (int j = 0; j < ntiles; j++) {
      const int b = j & 1;
      // warp-uniform: tcgen05.ld needs the whole warp
      if (!__all_sync(kFull, *abort_flag == 0 && tc::mbar_wait(done + b, (uint32_t)((j >> 1) & 1)))) {
        *abort_flag = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t lane_base =
          tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * TN + cbeg);
      const int jbase = j * TN + cbeg;
#pragma unroll 1
      for (int c0 = 0; c0 < TN / kEsplit; c0 += 32) {
        float acc[32];
        tc::tmem_ld_32x32(lane_base + (uint32_t)c0, acc);
#pragma unroll
        for (int jj = 0; jj < 32; jj++) {
          if (acc[jj] > best[jj & 3]) {
            best[jj & 3] = acc[jj];
            bidx[jj & 3] = jbase + c0 + jj;
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(empty + b);
    }
    // merge the chains: largest value, then lowest index
    bv = best[0];
    bi = bidx[0];
#pragma unroll
    for (int c = 1; c < 4; c++)
      if (best[c] > bv || (best[c] == bv && bidx[c] < bi)) {
        bv = best[c];
        bi = bidx[c];
      }
    pv[part * kTileM + quad * 32 + lane] = bv;
    pi[part * kTileM + quad * 32 + lane] = bi;
  }
  tc::fence_before_sync();
  __syncthreads();
  const bool ok = *abort_flag == 0;
  int64_t gr = n;
  int c = 0;
  if (warp < 4) {
    const int rrow = warp * 32 + lane;
    for (int q = 1; q < kEsplit; q++) {
      const float ov = pv[q * kTileM + rrow];
      const int oi = pi[q * kTileM + rrow];
      if (ov > bv || (ov == bv && oi < bi)) bv = ov, bi = oi;
    }
    gr = row0 + rrow;
    // a point whose values are all NaN keeps index 0: a valid cluster
    c = ok && bi < R ? bi : 0;
    if (gr < n) cl[gr] = c;
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  if (warp == 0) {
    __syncwarp();
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, ncols);
  }
  // the exact FP32 distance to the chosen representative, summed in
  // dimension order with fma (dist2_rows_rt): the only one the bounds use
  if (gr < n) dr[gr] = sqrtf(dist2_rows_rt(rows + gr * dp4, reps + (int64_t)c * dp4, dp4));
}

bool assign_tc_supported(int d) { return d >= 16 && d <= 256; }

// contraction depth: the coordinates and three norm columns, in MMA steps
static int assign_kd(int d) { return (d + 3 + 15) / 16 * 16; }

size_t assign_tc_scratch_bytes(int R, int d) {
  const int Rpad = (R + kTileN - 1) / kTileN * kTileN;
  return tc::tile_bytes(Rpad, assign_kd(d)) + 256;
}

int launch_assign_tc(const float4 *rows, int64_t n, int dp4, int d, const float4 *reps, int R,
                     void *scratch, int32_t *cl, float *dr, int *err, cudaStream_t s) {
  if (n == 0) return KNN_OK;
  const int KD = assign_kd(d);
  const int Rpad = (R + kTileN - 1) / kTileN * kTileN;
  __nv_bfloat16 *tiles = static_cast<__nv_bfloat16 *>(scratch);
  reps_to_bf16_tiles_kernel<<<(Rpad + 127) / 128, 128, 0, s>>>(reps, R, dp4, d, KD, Rpad, tiles);
  KNN_LAUNCH_CHECK();
  // representative tiles of 128 rows: a CTA then holds 256 TMEM columns and
  // two CTAs share an SM (measured faster than 256-row tiles with one CTA
  // per SM, with either 8 or 16 epilogue warps)
  const int TN = KNN_ASSIGN_TN;
  const size_t need = tc::tile_bytes(kTileM, KD) + (size_t)kStages * tc::tile_bytes(TN, KD) +
                      (kStages + 4) * sizeof(uint64_t) + 16 + (size_t)kEsplit * kTileM * 8;
  // a CTA holds 2 x TN TMEM columns: with TN = 256 that is all 512, so at
  // most one CTA per SM (over 114 KB each), with TN = 128 at most two
  const size_t smem = std::max<size_t>(need, TN == kTileN ? 116 * 1024 : 80 * 1024);
  KNN_CUDA_TRY(cudaFuncSetAttribute(assign_tc_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  KNN_CUDA_TRY(cudaFuncSetAttribute(assign_tc_kernel,
                                    cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
  const int64_t blocks = (n + kTileM - 1) / kTileM;
  assign_tc_kernel<<<(unsigned)blocks, kAssignThreads, smem, s>>>(
      rows, n, dp4, d, KD, TN, tiles, Rpad / TN, reps, R, cl, dr, err);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}

}  // namespace knnsweet

// Test hook (not part of the public ABI): nearest representative of every
// row on the tensor cores (use_tc != 0) or with the FP32 CUDA-core kernel,
// on device buffers; rows and reps are row-major n x d / R x d floats.
extern "C" int knnsweet_test_assign(const float *rows, int64_t n, const float *reps, int R,
                                    int d, int use_tc, int32_t *cl, float *dr) {
  using namespace knnsweet;
  const int dp4 = (d + 3) / 4;
  float4 *pr = nullptr, *rr = nullptr;
  void *scratch = nullptr;
  int *err = nullptr;
  int rc = KNN_OK;
  cudaStream_t s = 0;
  auto fail = [&](cudaError_t e) {
    set_error("%s", cudaGetErrorString(e));
    rc = KNN_ECUDA;
  };
  cudaError_t e = cudaMalloc(&pr, sizeof(float4) * n * dp4);
  if (e == cudaSuccess) e = cudaMalloc(&rr, sizeof(float4) * (size_t)R * dp4);
  if (e == cudaSuccess) e = cudaMalloc(&scratch, assign_tc_scratch_bytes(R, d));
  if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(int));
  if (e != cudaSuccess) fail(e);
  if (rc == KNN_OK) rc = launch_pack_rows(rows, n, d, dp4, pr, s);
  if (rc == KNN_OK) rc = launch_pack_rows(reps, R, d, dp4, rr, s);
  if (rc == KNN_OK) {
    if (use_tc) {
      rc = assign_tc_supported(d) ? launch_assign_tc(pr, n, dp4, d, rr, R, scratch, cl, dr, err, s)
                                  : KNN_EINVAL;
    } else {
      rc = launch_assign(pr, n, dp4, rr, R, cl, dr, s);
    }
  }
  if (rc == KNN_OK) {
    e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) fail(e);
    else if (h) {
      set_error("tensor-core assignment timed out");
      rc = KNN_ETIMEOUT;
    }
  }
  cudaFree(pr);
  cudaFree(rr);
  cudaFree(scratch);
  cudaFree(err);
  return rc;
}
