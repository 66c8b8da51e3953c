// sharded.cu -- the join over several GPUs of one process, by query ranges.
//
// Queries are independent (each one's k nearest references depend on nothing
// else), so the path shards with no data-path collective: every listed device
// builds the reference index (the same options and seed, so the same index)
// and answers one contiguous range of the queries, writing its rows of the
// host result.  One host thread per shard; shards listing the same device run
// concurrently on their own streams.  The reference program has no
// counterpart (it uses one GPU, src/knnjoin.cu:983-1172).
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace knnsweet {
std::string &error_buffer();
int check_sizes(int64_t m, int64_t n, int32_t d, int32_t k);
}  // namespace knnsweet

namespace {

struct Shard {
  int device = 0;
  int64_t q0 = 0, m = 0;
  int rc = KNN_OK;
  std::string err;
  knn_stats st{};
};

// One shard on its device: copy the references and the shard's queries in,
// build the index, query it, copy the rows back.
void run_shard(Shard *sh, const float *q, const float *r, int64_t n, int32_t d, int32_t k,
               int32_t *out_idx, float *out_dist, const knn_options *opt, bool want_stats) {
  auto cuda_fail = [&](cudaError_t e, const char *what) {
    sh->rc = KNN_ECUDA;
    sh->err = std::string(what) + ": " + cudaGetErrorString(e);
  };
  cudaError_t e = cudaSetDevice(sh->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  cudaStream_t s = nullptr;
  e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(e, "stream creation");
  float *dr = nullptr, *dq = nullptr, *dd = nullptr;
  int32_t *di = nullptr;
  knn_index *ix = nullptr;
  const size_t rows = (size_t)sh->m * (size_t)k;
  e = cudaMallocAsync(&dr, sizeof(float) * (size_t)n * d, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&dq, sizeof(float) * (size_t)sh->m * d, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&di, sizeof(int32_t) * rows, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&dd, sizeof(float) * rows, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dr, r, sizeof(float) * (size_t)n * d, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dq, q + sh->q0 * d, sizeof(float) * (size_t)sh->m * d,
                        cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    cuda_fail(e, "device buffers");
  } else {
    // device time of the shard: index build + query (events on its stream)
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (want_stats && (cudaEventCreate(&ev[0]) != cudaSuccess ||
                       cudaEventCreate(&ev[1]) != cudaSuccess)) {
      cudaGetLastError();
      want_stats = false;
    }
    if (want_stats) cudaEventRecord(ev[0], s);
    int rc = knn_index_build(dr, n, d, opt, &ix, s);
    if (rc == KNN_OK)
      rc = knn_index_query(ix, dq, sh->m, k, di, dd, opt, want_stats ? &sh->st : nullptr, s);
    if (want_stats) {
      cudaEventRecord(ev[1], s);
      float ms = 0.0f;
      if (rc == KNN_OK && cudaEventSynchronize(ev[1]) == cudaSuccess &&
          cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) {
        sh->st.ms_build += ms - sh->st.ms_total;  // + the index build
        sh->st.ms_total = ms;
      }
    }
    for (cudaEvent_t x : ev)
      if (x) cudaEventDestroy(x);
    if (rc != KNN_OK) {
      sh->rc = rc;
      sh->err = knn_last_error();
    } else {
      e = cudaMemcpyAsync(out_idx + sh->q0 * k, di, sizeof(int32_t) * rows,
                          cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_dist + sh->q0 * k, dd, sizeof(float) * rows,
                            cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) cuda_fail(e, "join");
    }
  }
  cudaStreamSynchronize(s);
  if (ix) knn_index_free(ix);
  cudaFreeAsync(dr, s);
  cudaFreeAsync(dq, s);
  cudaFreeAsync(di, s);
  cudaFreeAsync(dd, s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
}

}  // namespace

extern "C" int knn_join_sharded(const float *q, int64_t m, const float *r, int64_t n,
                                int32_t d, int32_t k, int32_t *out_idx, float *out_dist,
                                const knn_options *opt, const int32_t *devices, int32_t ndev,
                                knn_stats *st) {
  using namespace knnsweet;
  error_buffer().clear();
  if (st) memset(st, 0, sizeof *st);
  const int rc0 = check_sizes(m, n, d, k);
  if (rc0 != KNN_OK) return rc0;
  if (!devices || ndev <= 0 || ndev > 4096) {
    set_error("devices must list 1 to 4096 device ids");
    return KNN_EINVAL;
  }
  if (m == 0) return KNN_OK;
  if (!q || !out_idx || !out_dist || (n > 0 && !r)) {
    set_error("null pointer argument");
    return KNN_EINVAL;
  }
  if (n == 0) {  // no references: every slot is empty, as in knn_join
    for (int64_t i = 0; i < m * k; i++) {
      out_idx[i] = -1;
      out_dist[i] = std::numeric_limits<float>::infinity();
    }
    return KNN_OK;
  }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) {
    set_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return KNN_ECUDA;
  }
  for (int i = 0; i < ndev; i++)
    if (devices[i] < 0 || devices[i] >= count) {
      set_error("device %d is not one of the %d devices", devices[i], count);
      return KNN_EINVAL;
    }
  // contiguous query ranges, as even as the count allows
  std::vector<Shard> sh(ndev);
  for (int i = 0; i < ndev; i++) {
    sh[i].device = devices[i];
    sh[i].q0 = m * i / ndev;
    sh[i].m = m * (i + 1) / ndev - sh[i].q0;
  }
  std::vector<std::thread> th;
  for (int i = 0; i < ndev; i++)
    if (sh[i].m > 0)
      th.emplace_back(run_shard, &sh[i], q, r, n, d, k, out_idx, out_dist, opt, st != nullptr);
  for (auto &t : th) t.join();
  for (int i = 0; i < ndev; i++)
    if (sh[i].rc != KNN_OK) {
      set_error("shard %d (device %d): %s", i, sh[i].device, sh[i].err.c_str());
      return sh[i].rc;
    }
  if (st) {
    for (const Shard &s : sh) {
      if (s.m == 0) continue;
      st->dist_evals += s.st.dist_evals;
      st->clusters_visited += s.st.clusters_visited;
      st->clusters_pruned += s.st.clusters_pruned;
      st->fp64_rechecks += s.st.fp64_rechecks;
      st->topk_candidates += s.st.topk_candidates;
      st->topk_merges += s.st.topk_merges;
      st->ms_build = s.st.ms_build > st->ms_build ? s.st.ms_build : st->ms_build;
      st->ms_search = s.st.ms_search > st->ms_search ? s.st.ms_search : st->ms_search;
      st->ms_total = s.st.ms_total > st->ms_total ? s.st.ms_total : st->ms_total;
      st->qreps_used += s.st.qreps_used;
      st->sreps_used = s.st.sreps_used;
      st->kernels_launched += s.st.kernels_launched;
      st->refine_fallbacks += s.st.refine_fallbacks;
      st->band_queries += s.st.band_queries;
    }
    st->pairs_total = m * n;
    st->pairs_pruned = st->pairs_total - st->dist_evals;
  }
  return KNN_OK;
}
