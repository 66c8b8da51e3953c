// pipeline.cuh -- the stages of one join shared by the entry points
// (api.cu: single device; sharded.cu: several devices): scratch arenas, the
// device counter layout, the reference and query sides and the search.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace knnsweet {

#define KNN_TRY(expr)        \
  do {                       \
    int rc_ = (expr);        \
    if (rc_ != KNN_OK) return rc_; \
  } while (0)

// Stream-ordered scratch: every allocation is released on the same stream
// when the arena goes out of scope.
class Arena {
 public:
  explicit Arena(cudaStream_t s) : s_(s) {}
  ~Arena() {
    for (void *p : ptrs_) cudaFreeAsync(p, s_);
  }
  Arena(const Arena &) = delete;
  Arena &operator=(const Arena &) = delete;

  // Hands the allocations made so far to the caller: they outlive the arena.
  std::vector<void *> take() {
    std::vector<void *> out;
    out.swap(ptrs_);
    return out;
  }

  template <class T>
  int alloc(T **out, size_t count) {
    *out = nullptr;
    if (count == 0) count = 1;
    if (!pool_) {
      int rc = scratch_pool(&pool_);
      if (rc != KNN_OK) return rc;
    }
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, count * sizeof(T), pool_, s_);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation of %zu bytes failed: %s", count * sizeof(T),
                cudaGetErrorString(e));
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

// Device counters of one call, zeroed at its start.
enum CtrSlot {
  kCtrWork = 0,                         // scan work counter
  kCtrScan = 1,                         // the scan statistics (kScanCounters)
  kCtrErr = kCtrScan + kScanCounters,   // device error flag (bounded waits)
  kCtrTileWork,                         // tile-search tile counter
  kCtrTile,                             // tile-search statistics (4)
  kCtrFallback = kCtrTile + 4,          // slots the tile search leaves to the scan
  kCtrUnres,                            // queries left to the band kernel
  kCtrInexactQ,                         // the query side is not small integers
  kCtrCount
};

// One clustered point set.
struct ClusterSet {
  int R = 0;
  float4 *reps = nullptr;     // R x dp4s
  int32_t *rep_rows = nullptr;
  uint64_t *skeys = nullptr;  // n sorted (cluster, distance) keys
  int32_t *perm = nullptr;    // sorted position -> input row
  int32_t *off = nullptr;     // R + 1
};

// Host destination of the result for the host-buffer entry point: the scan
// then runs in row chunks and each chunk's rows are copied back on `copy`
// while the next chunk is computed.  `done` tells whether the copies were
// enqueued (otherwise the caller copies the whole result).
struct HostSink {
  int32_t *idx;
  float *dist;
  cudaStream_t copy;
  bool done;
};

// The reference side of a join: representatives, clusters, the
// cluster-contiguous rows and their bounds.  Depends only on the reference
// set and the options that shape its clusters.
struct RefSide {
  int64_t n = 0;
  int d = 0, dp4s = 0, tmpl = 0, Rs = 0;
  bool idx_in_row = false;
  ClusterSet sset;
  const float4 *Rp = nullptr;  // packed rows, original order
  float4 *srows = nullptr;     // cluster-contiguous rows
  float *sdist = nullptr, *cmin = nullptr, *cmax = nullptr;
  int32_t *sidx = nullptr;
  int *inexact = nullptr;      // device flag: 0 when the rows are small integers
};

// The query side of a join against a built reference side: query rows,
// query clusters, representative distances, the k-th bounds and the
// surviving reference clusters of every query cluster.
struct QuerySide {
  int Rq = 0;
  const float4 *Qp = nullptr;  // query rows (packed), original order
  ClusterSet qset;             // qset.perm: slot -> query row; qset.off: slots of a cluster
  const int *inexact = nullptr;
  float *qrad = nullptr, *drr = nullptr, *theta0 = nullptr;
  int32_t *slot_cl = nullptr, *rlist = nullptr, *rlen = nullptr;
  float2 *clb = nullptr;  // per list chunk: first d(Rq, Rs), largest radius from it on
};

// Argument and option ranges shared by every entry point.
int check_sizes(int64_t m, int64_t n, int32_t d, int32_t k);
int check_options(const knn_options *opt, knn_options *o);
// Representative count for n points when the caller passes 0.
int default_reps(int64_t n);
// Number of query representatives for m queries.
int query_rep_count(const knn_options &o, int64_t m, int d, int k, bool self, int Rs);
// Builds the reference side of reference rows r (device); the arrays it keeps
// come from `keep`, scratch from `tmp`.
int build_ref_side(Arena &keep, Arena &tmp, const float *r, int64_t n, int d, int Rs,
                   const knn_options &o, bool copy_rows, int *dev_err, cudaStream_t s,
                   RefSide *R);
// Builds the query side of queries q (device) against R (share: the join is a
// self-join using R's clusters).
int build_query_side(const RefSide &R, bool share, const float *q, int64_t m, int32_t k,
                     const knn_options &o, Arena &ar, unsigned long long *ctr, cudaStream_t s,
                     QuerySide *Q);
// Searches the query clusters c0 .. c1-1 (slots slot0 .. slot0+nslot-1).
int search_clusters(const RefSide &R, const QuerySide &Q, int64_t m, int32_t k, int c0, int c1,
                    int64_t slot0, int64_t nslot, int32_t *out_idx, float *out_dist,
                    const knn_options &o, cudaStream_t s, HostSink *sink, Arena &ar,
                    unsigned long long *ctr);
// Adds the device counters of one call to `st` (synchronises `s`).
int read_stats(const unsigned long long *ctr, cudaStream_t s, knn_stats *st);

}  // namespace knnsweet
