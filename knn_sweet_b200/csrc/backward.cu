// backward.cu -- gradient of a loss over kNN pairs (no reference
// counterpart: the reference computes no gradient).
//
// For every pair (i, j = idx[i*k + t]) with upstream gradient g on the
// squared distance |q_i - r_j|^2:
//     grad_q[i] += 2 g (q_i - r_j)        grad_r[j] -= 2 g (q_i - r_j)
// One thread per (query, coordinate): the k pairs of the query are summed in
// registers and added to grad_q once; the reference side is scattered with
// float atomics (the neighbour sets are constants of the forward pass).
#include "common.cuh"

namespace knnsweet {

__global__ void knn_backward_kernel(const float *__restrict__ q, int64_t m,
                                    const float *__restrict__ r, int64_t n,
                                    int d, int k,
                                    const int32_t *__restrict__ idx,
                                    const float *__restrict__ g,
                                    float *__restrict__ gq,
                                    float *__restrict__ gr) {
  const int64_t total = m * d;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / d;
    const int c = (int)(e - i * d);
    const float qi = q[e];
    float acc = 0.0f;
    for (int t = 0; t < k; t++) {
      const int32_t j = idx[i * k + t];
      if (j < 0 || j >= n) continue;
      const float diff = qi - r[(int64_t)j * d + c];
      const float v = 2.0f * g[i * k + t] * diff;
      acc += v;
      if (gr) atomicAdd(gr + (int64_t)j * d + c, -v);
    }
    gq[e] += acc;
  }
}

}  // namespace knnsweet

using namespace knnsweet;

extern "C" int knn_backward_device(const float *q, int64_t m, const float *r,
                                   int64_t n, int32_t d, int32_t k,
                                   const int32_t *idx, const float *grad_dist2,
                                   float *grad_q, float *grad_r, void *stream) {
  error_buffer().clear();
  if (d <= 0 || k <= 0 || m < 0 || n < 0) {
    set_error("backward: bad sizes");
    return KNN_EINVAL;
  }
  if (m == 0) return KNN_OK;
  if (!q || !r || !idx || !grad_dist2 || !grad_q) {
    set_error("backward: null pointer argument");
    return KNN_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t total = m * d;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  knn_backward_kernel<<<(int)blocks, 256, 0, s>>>(q, m, r, n, d, k, idx, grad_dist2,
                                                  grad_q, grad_r);
  KNN_LAUNCH_CHECK();
  return KNN_OK;
}
