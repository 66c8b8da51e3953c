// kernels.cuh -- launcher declarations shared by the translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// A query (a tile of queries) stops walking its candidate list where the
// rest of it is prunable as a whole (1), or tests every entry (0).
#ifndef KNN_CHUNK_EXIT
#define KNN_CHUNK_EXIT 1
#endif

namespace knnsweet {

// Statistics the scan kernels accumulate (ScanArgs::counters): distance
// evaluations, clusters visited, clusters pruned, candidates pushed, top-k
// merges, FP64 distances of the k-th boundary, queries the band kernel
// settled.
constexpr int kScanCounters = 7;

// Arguments of the per-query scan.
struct ScanArgs {
  const float4 *qrows;      // m x dp4, original query order
  const int32_t *qorder;    // slot -> query row (grouped by query cluster)
  const int32_t *slot_cl;   // slot -> query cluster
  int64_t m;
  int d, dp4, dp4_tmpl, k;
  bool idx_in_row;          // srows carry the index in their last pad float
  bool squared;             // write squared distances instead of distances
  const float4 *sreps;      // Rs x dp4 reference representatives
  const float4 *srows;      // n x dp4, cluster-contiguous, ascending d(s,Rs)
  const float *sdist;       // n: d(s, Rs) in the same order
  const int32_t *sidx;      // n: original reference row
  const int32_t *soff;      // Rs + 1 cluster offsets
  const float *cmin, *cmax; // Rs: smallest / largest member distance
  const float *theta0;      // Rq: initial k-th bound per query cluster
  const float *qrad;        // Rq: query cluster radius (the one theta0 used) ...
  const uint64_t *qkeys;    // ... and slot -> (cluster, d(q, Rq)) sort key: a
                            // query's own bound theta0 - (rq - d(q,Rq)); null: theta0
  const int32_t *rlist;     // Rq x Rs surviving clusters, nearest first
  const int32_t *rlen;      // Rq
  const float2 *clb;        // optional (null: none): per query cluster and 32
                            // list entries, x = d(Rq, Rs) of the chunk's first
                            // entry, y = the largest radius from that entry on
  int clb_stride;           // chunks per query cluster in clb
  const int64_t *rl_base;   // batched form: start of each query cluster's list
                            // in rlist (null: qc * Rs)
  const int64_t *qc_ref_base;  // batched form: subtracted from every output
                               // index of query cluster qc (null: 0)
  const int32_t *slot_list;    // optional: scan only these slots ...
  const unsigned *slot_count;  // ... *slot_count of them (device count);
  int64_t slot_base;           // without a list: slots slot_base .. + m - 1
  int Rs;
  int64_t n_ref;            // reference points (0: unknown); with Rs it gives
                            // the mean cluster size the scan variant is chosen by
  const float4 *rrows;      // n x dp4 reference rows, original order (the
                            // FP64 re-check of the k-th boundary)
  const int *inexact_r;     // device flags of the two sides, 0 when every
  const int *inexact_q;     // coordinate is a small integer (then FP32
                            // distances are exact and rank like FP64)
  int32_t *out_idx;         // m x k
  float *out_dist;          // m x k
  int32_t *unres_slot;      // room for every slot of the launch: queries
                            // whose boundary the band kernel settles ...
  unsigned *unres_count;    // ... and their number (zeroed by launch_scan)
  unsigned long long *work_counter;  // zeroed before launch
  unsigned long long *counters;      // kScanCounters statistics (or null)
};

int launch_pack_rows(const float *src, int64_t n, int d, int dp4, float4 *dst,
                     cudaStream_t s);
// Raises *inexact unless every value of x[0..count) is an integer small enough
// that FP32 squared distances in dimension d are exact.
int launch_exact_check(const float *x, int64_t count, int d, int *inexact, cudaStream_t s);
// Estimated search work per query cluster (for partitioning across devices).
int launch_cluster_work(const float *drr, int Rq, int Rs, const float *qrad, const float *theta0,
                        const int32_t *qoff, const int32_t *rlist, const int32_t *rlen,
                        const int32_t *soff, const float *sdist, long long *work,
                        cudaStream_t s);
int launch_rep_select(const float4 *rows, int dp4, const int32_t *cand_dev,
                      int R, int trials, uint32_t *score_dev, float4 *reps,
                      int32_t *rep_rows, cudaStream_t s);
int launch_assign(const float4 *rows, int64_t n, int dp4, const float4 *reps,
                  int R, int32_t *cl, float *dr, cudaStream_t s);
// Tensor-core assignment (assign_tc.cu): rows of d >= 16 floats.
bool assign_tc_supported(int d);
size_t assign_tc_scratch_bytes(int R, int d);
int launch_assign_tc(const float4 *rows, int64_t n, int dp4, int d, const float4 *reps, int R,
                     void *scratch, int32_t *cl, float *dr, int *err, cudaStream_t s);
size_t cluster_sort_temp_bytes(int64_t n, int R);
int launch_centroids(const float4 *rows, int dp4, const int32_t *perm, const int32_t *off, int R,
                     float4 *reps, cudaStream_t s);
int launch_split_clusters(const float4 *rows, int dp4, const int32_t *perm, const int32_t *off,
                          const uint64_t *skeys, int R, float4 *reps, cudaStream_t s);
int launch_cluster_sort(const int32_t *cl, const float *dr, int64_t n, int R,
                        uint64_t *keys, int32_t *vals, uint64_t *skeys,
                        int32_t *perm, void *temp, size_t temp_bytes,
                        cudaStream_t s);
size_t chunk_slots_temp_bytes(int64_t m, int nchunks);
int launch_chunk_slots(const int32_t *qorder, int64_t m, int first, int chunk_rows, int nchunks,
                       uint32_t *keys, uint32_t *keys_out, int32_t *vals, int32_t *slots,
                       void *temp, size_t temp_bytes, cudaStream_t s);
int launch_cluster_layout(const uint64_t *skeys, const int32_t *perm, int64_t n,
                          const float4 *rows, int dp4, bool idx_in_row,
                          float4 *srows, float *sdist, int32_t *sidx,
                          cudaStream_t s);
int launch_cluster_offsets(const uint64_t *skeys, int64_t n, int R, int32_t *off,
                           cudaStream_t s);
int launch_cluster_minmax(const int32_t *off, const float *sdist, int R,
                          float *cmin, float *cmax, cudaStream_t s);
int launch_query_clusters(const uint64_t *skeys, const int32_t *off, int64_t m,
                          int R, float *qrad, int32_t *slot_cl, cudaStream_t s);
int launch_rep_dist(const float4 *qreps, int Rq, const float4 *sreps, int Rs,
                    int dp4, float *drr, cudaStream_t s);
int launch_bounds_filter(const float *drr, int Rq, int Rs, const float *qrad,
                         const int32_t *qoff, const int32_t *soff,
                         const float *sdist, const float *scmax, int k, int d,
                         float *theta0, int32_t *rlist, int32_t *rlen,
                         float2 *clb, cudaStream_t s);
int launch_scan(const ScanArgs &a, int num_sms, cudaStream_t s);

// Arguments of the BF16 tensor-core tile search with FP32 re-ranking
// (tile_search.cu).
struct TileArgs {
  const float4 *qrows;       // m x dp4 queries, original order
  int dp4, d, KD;            // row stride (float4), width, padded MMA K
  const int32_t *qorder;     // slot -> query row (grouped by query cluster)
  const int32_t *tiles;      // per tile: {query cluster, first slot, count,
                             // slot of the centre point}
  const int32_t *ntiles;     // device: number of tiles
  const float4 *srows;       // n x dp4 reference rows, cluster-contiguous
  const int32_t *sidx;       // n: original reference row
  const float4 *rrows;       // n x dp4 reference rows, original order
  const int32_t *soff;       // Rs + 1
  const float *sdist;        // n: d(s, Rs), ascending within each cluster
  const float *cmin, *cmax;  // Rs: smallest / largest member distance
  const float4 *sreps;       // Rs x dp4 reference representatives
  const int32_t *rlist;      // Rq x Rs surviving clusters, nearest first
  const int32_t *rlen;       // Rq
  int Rs;
  const float2 *clb;         // optional: per list chunk, as ScanArgs::clb
  int clb_stride;
  const uint64_t *qkeys;     // slot -> (cluster, d(q, Rq)) key (with clb)
  const float *theta0;       // Rq: k-th distance bound per query cluster
  int k, cap, P;             // k; buffer entries per query; sort scratch (pow2)
  bool squared;
  float2 *buf_lu;            // grid x 128 x cap: (lower, upper) bound pairs
  int32_t *buf_pos;          // grid x 128 x cap: cluster-layout positions
  int32_t *out_idx;
  float *out_dist;
  unsigned long long *work;  // tile counter, zeroed
  int32_t *fb_slots;         // slots left to the FP32 scan
  unsigned *fb_count;
  int *err;                  // set when a bounded wait gives up
  unsigned long long *counters;  // [tensor pairs, refined, fp64 rechecks, fallbacks]
};
bool tile_search_supported(int d, int k, int margin);
int tile_search_geometry(int d, int k, int margin, int num_sms, int *grid, int *cap, int *P,
                         size_t *smem);
// Tiles of the query clusters c_base .. c_base + Rq - 1 (qoff points at
// c_base's offset; the tiles carry absolute cluster ids and slots).
int launch_tile_list(const int32_t *qoff, int Rq, int c_base, int32_t *tiles, int32_t *ntiles,
                     cudaStream_t s);
int launch_tile_search(const TileArgs &a, int grid, size_t smem, cudaStream_t s);

// The calling thread's two streams for host-buffer calls (cached per device,
// idle between calls).
int host_streams(cudaStream_t *s, cudaStream_t *cs);

}  // namespace knnsweet
