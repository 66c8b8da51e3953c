// assign_tc.cu -- nearest representative on the tensor cores (tcgen05).
//
// For rows wide enough to be a dense contraction (d >= 16) the assignment of
// every point to its nearest representative (findQCluster / findTCluster,
// src/knnjoin.cu:64-97, over the cuBLAS distance matrix of knnjoin.cu:270-342)
// is an n x R x d GEMM with an arg-min epilogue:
//     argmin_j  |r_j|^2 - 2 p . r_j
// computed from BF16-rounded points and representatives with FP32 accumulation
// in TMEM.  The choice only has to be approximately nearest: the pruning
// bounds need the exact distance to whichever representative is chosen, and
// that distance is recomputed in FP32 afterwards (exact_rep_dist_kernel).
//
// One CTA (one warpgroup, 128 threads) owns 128 points: it converts them to
// BF16 into shared memory in the core-matrix layout of tc_common.cuh, then for
// every tile of 256 representatives (pre-converted once) thread 0 issues
// KD/16 MMAs (M = 128, N = 256, K = 16) into a 256-column TMEM accumulator and
// commits to an mbarrier; each warp then reads its 32 rows back
// (tcgen05.ld 32x32b) and keeps a running arg-min per row.  Every wait is
// bounded; on timeout the CTA flags the error, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_common.cuh"

namespace knnsweet {

namespace {
constexpr int kTileM = 128;  // points per CTA (TMEM lanes)
constexpr int kTileN = 256;  // representatives per MMA (TMEM columns)
}  // namespace

// Representatives -> BF16 tiles of kTileN rows in the core-matrix layout, and
// their squared norms (of the rounded values); padding rows get norm +inf so
// they never win the arg-min.
__global__ void reps_to_bf16_tiles_kernel(const float4 *__restrict__ reps, int R, int dp4,
                                          int d, int KD, int Rpad,
                                          __nv_bfloat16 *__restrict__ tiles,
                                          float *__restrict__ rnorm) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Rpad) return;
  unsigned char *tile = reinterpret_cast<unsigned char *>(tiles) +
                        (size_t)(r / kTileN) * tc::tile_bytes(kTileN, KD);
  const int rr = r % kTileN;
  float nrm = 0.0f;
  for (int k0 = 0; k0 < KD; k0 += 8) {
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int k = k0 + e;
      float x = 0.0f;
      if (r < R && k < d) {
        const float4 c = reps[(size_t)r * dp4 + (k >> 2)];
        x = (k & 3) == 0 ? c.x : (k & 3) == 1 ? c.y : (k & 3) == 2 ? c.z : c.w;
      }
      v[e] = __float2bfloat16_rn(x);
      const float xr = __bfloat162float(v[e]);
      nrm = __fmaf_rn(xr, xr, nrm);
    }
    *reinterpret_cast<uint4 *>(tile + tc::tile_offset(rr, k0, KD)) =
        *reinterpret_cast<const uint4 *>(v);
  }
  rnorm[r] = r < R ? nrm : __int_as_float(0x7f800000);
}

__global__ void __launch_bounds__(128)
    assign_tc_kernel(const float4 *__restrict__ rows, int64_t n, int dp4, int d, int KD,
                     const __nv_bfloat16 *__restrict__ rep_tiles,
                     const float *__restrict__ rnorm, int ntiles_r,
                     int32_t *__restrict__ cl, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sa = smem;                                   // kTileM x KD
  unsigned char *sb = sa + tc::tile_bytes(kTileM, KD);        // kTileN x KD
  float *srn = reinterpret_cast<float *>(sb + tc::tile_bytes(kTileN, KD));
  uint64_t *mbar = reinterpret_cast<uint64_t *>(srn + kTileN);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t row0 = (int64_t)blockIdx.x * kTileM;

  if (warp == 0) tc::tmem_alloc(tmem_slot, kTileN);
  if (tid == 0) tc::mbar_init(mbar, 1);
  // points -> BF16 core-matrix tile (thread = one row at a time, 8 columns)
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
      }
      v[e] = __float2bfloat16_rn(x);
    }
    *reinterpret_cast<uint4 *>(sa + tc::tile_offset(r, k0, KD)) =
        *reinterpret_cast<const uint4 *>(v);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const uint32_t idesc = tc::make_idesc_bf16(kTileM, kTileN);
  const uint32_t a_base = tc::smem_u32(sa), b_base = tc::smem_u32(sb);
  const uint32_t sbo = (uint32_t)KD * 16;  // next 8-row group
  float best = __int_as_float(0x7f800000);
  int best_j = 0;
  bool ok = true;
  const size_t btile = tc::tile_bytes(kTileN, KD);

  for (int rt = 0; rt < ntiles_r && ok; rt++) {
    // representative tile -> shared memory (contiguous copy) + its norms
    const uint4 *src = reinterpret_cast<const uint4 *>(
        reinterpret_cast<const unsigned char *>(rep_tiles) + (size_t)rt * btile);
    uint4 *dst = reinterpret_cast<uint4 *>(sb);
    for (int i = tid; i < (int)(btile / 16); i += blockDim.x) dst[i] = src[i];
    for (int i = tid; i < kTileN; i += blockDim.x) srn[i] = rnorm[(size_t)rt * kTileN + i];
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      for (int s = 0; s < KD / 16; s++) {
        const uint64_t ad = tc::make_desc(a_base + 256u * s, 128u, sbo);
        const uint64_t bd = tc::make_desc(b_base + 256u * s, 128u, sbo);
        tc::mma_bf16(tmem, ad, bd, idesc, s > 0);
      }
      tc::mma_commit(mbar);
    }
    ok = tc::mbar_wait(mbar, (uint32_t)(rt & 1));
    ok = __syncthreads_and(ok) != 0;  // one decision for the whole CTA
    if (!ok) break;
    tc::fence_after_sync();
    // this warp's 32 rows, 32 columns at a time
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < kTileN; c += 32) {
      float acc[32];
      tc::tmem_ld_32x32(lane_base + (uint32_t)c, acc);
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const float v = __fmaf_rn(-2.0f, acc[j], srn[c + j]);
        if (v < best) {
          best = v;
          best_j = rt * kTileN + c + j;
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();  // TMEM and the B tile are reused by the next step
    tc::fence_after_sync();
  }
  if (!ok && lane == 0) atomicExch(err, 1);
  const int64_t gr = row0 + warp * 32 + lane;
  if (gr < n) cl[gr] = ok ? best_j : 0;  // always a valid representative
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTileN);
}

// Exact FP32 distance of every point to its chosen representative.
__global__ void exact_rep_dist_kernel(const float4 *__restrict__ rows, int64_t n, int dp4,
                                      const float4 *__restrict__ reps,
                                      const int32_t *__restrict__ cl, float *__restrict__ dr) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dr[i] = sqrtf(dist2_rows_rt(rows + i * dp4, reps + (int64_t)cl[i] * dp4, dp4));
}

bool assign_tc_supported(int d) { return d >= 16 && d <= 256; }

size_t assign_tc_scratch_bytes(int R, int d) {
  const int KD = (d + 15) / 16 * 16;
  const int Rpad = (R + kTileN - 1) / kTileN * kTileN;
  return tc::tile_bytes(Rpad, KD) + 256 + (size_t)Rpad * sizeof(float) + 256 + 256;
}

int launch_assign_tc(const float4 *rows, int64_t n, int dp4, int d, const float4 *reps, int R,
                     void *scratch, int32_t *cl, float *dr, int *err, cudaStream_t s) {
  if (n == 0) return KNN_OK;
  const int KD = (d + 15) / 16 * 16;
  const int Rpad = (R + kTileN - 1) / kTileN * kTileN;
  unsigned char *p = static_cast<unsigned char *>(scratch);
  __nv_bfloat16 *tiles = reinterpret_cast<__nv_bfloat16 *>(p);
  float *rnorm = reinterpret_cast<float *>(p + ((tc::tile_bytes(Rpad, KD) + 255) & ~(size_t)255));
  reps_to_bf16_tiles_kernel<<<(Rpad + 127) / 128, 128, 0, s>>>(reps, R, dp4, d, KD, Rpad, tiles,
                                                               rnorm);
  KNN_LAUNCH_CHECK();
  // at least 100 KB, so that no more than two CTAs (2 x 256 TMEM columns of
  // the 512) share an SM and tcgen05.alloc never waits
  const size_t need = tc::tile_bytes(kTileM, KD) + tc::tile_bytes(kTileN, KD) +
                      kTileN * sizeof(float) + 16;
  const size_t smem = std::max<size_t>(need, 100 * 1024);
  KNN_CUDA_TRY(cudaFuncSetAttribute(assign_tc_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  KNN_CUDA_TRY(cudaFuncSetAttribute(assign_tc_kernel,
                                    cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
  const int64_t blocks = (n + kTileM - 1) / kTileM;
  assign_tc_kernel<<<(unsigned)blocks, 128, smem, s>>>(rows, n, dp4, d, KD, tiles, rnorm,
                                                       Rpad / kTileN, cl, err);
  KNN_LAUNCH_CHECK();
  exact_rep_dist_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, s>>>(
      rows, n, dp4, reps, cl, dr);
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
