/*
 * knnsweet.h -- C ABI of the B200-native exact kNN join (libknnsweet.so).
 *
 * The reference (knn_sweet) has no library interface: its boundary is the
 * `knnjoin` command line (src/knnjoin.cu:990-1001) over process globals
 * (include/common8.h:14-24), and its result is the array
 * `IndexDist knearest[query_nb*K]` (include/common8.h:37-40,
 * src/knnjoin.cu:1104, 1139-1141): for every query, in the original query
 * order, K pairs {source row index, Euclidean distance} in ascending distance.
 * Each entry point below replaces one piece of that contract; the comment on
 * each names the reference code it stands in for.
 *
 * Conventions
 *  - Points are row-major float32, `d` floats per row, rows packed (stride d).
 *  - Results are structure-of-arrays: out_idx[i*k + j] (int32, 0-based row of
 *    the reference set) and out_dist[i*k + j] (float32 Euclidean distance).
 *    The k indices of a query are the k nearest by (FP64 squared distance,
 *    index) -- exactly the set an FP64 brute-force join gives, ties at equal
 *    distance going to the lower reference index -- listed ascending by
 *    (FP32 squared distance, index).  knn_pack_indexdist() converts to the
 *    reference's interleaved {int index; float dist} layout.
 *  - When fewer than k reference points exist (k > n), the missing slots hold
 *    index -1 and distance +inf (the reference leaves them uninitialised).
 *  - Every call returns 0 (KNN_OK) or a negative KNN_E* code and never exits
 *    the process; knn_last_error() gives a message (per host thread).
 *  - Calls hold no global state and may run concurrently from several host
 *    threads; each device-buffer call uses the caller's stream, each
 *    host-buffer call two streams of the calling thread (created on its first
 *    host-buffer call on a device and reused; idle between calls).
 */
#ifndef KNNSWEET_H
#define KNNSWEET_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KNNSWEET_ABI_VERSION 2

/* Status codes (the reference prints and continues: src/knnjoin.cu:38-41). */
#define KNN_OK 0
#define KNN_EINVAL (-1)   /* bad argument: null pointer, d<=0, k<=0, sizes   */
#define KNN_ENOMEM (-2)   /* a device or host allocation failed              */
#define KNN_ECUDA (-3)    /* a CUDA runtime call or kernel launch failed     */
#define KNN_ETIMEOUT (-4) /* a bounded device wait gave up                   */
#define KNN_EINTERNAL (-5)/* a device-side consistency check failed          */

/* Precision forms. */
#define KNN_FP32 0        /* plain FP32 pruned join                          */
#define KNN_BF16_REFINE 1 /* BF16 tensor-core distance tiles with error
                             bounds, exact FP32 re-rank of the pairs the
                             bounds keep, FP64 re-check of the k-th boundary
                             (1 <= d <= 256; the neighbour set is the one an
                             FP64 join gives)                                */

/* Option flags. */
#define KNN_SQUARED_DIST 1 /* out_dist holds squared distances |q - r|^2     */
#define KNN_NO_TENSOR_CORES 2 /* CUDA-core FP32 kernels only (for comparison):
                             the point-to-representative assignment of rows
                             with d >= 16 otherwise runs on tcgen05 in BF16
                             (results are identical; only clusters differ)  */

/* Limits. */
#define KNN_MAX_K 1024    /* the reference allows K <= 1000 (knnjoin.cu:774) */
#define KNN_MAX_REPS 8192

/*
 * Options.  Defaults (knn_default_options): qreps = sreps = 0 meaning
 * "choose from the set size" (about sqrt(n)*1.6, at most 4096; the reference
 * takes them from argv[4], argv[5]: knnjoin.cu:997-998), seed = 2015
 * (knnjoin.cu:199, 226), rep_trials = 10 (knnjoin.cu:195), precision = FP32,
 * margin = 32, autotune = 1.
 */
typedef struct knn_options {
  int32_t qreps;      /* number of query representatives (query clusters)    */
  int32_t sreps;      /* number of reference representatives                 */
  uint32_t seed;      /* glibc srand() seed used to draw representative rows */
  int32_t rep_trials; /* random draws compared by pairwise spread            */
  int32_t precision;  /* KNN_FP32 or KNN_BF16_REFINE                          */
  int32_t margin;     /* BF16 form: re-ranking reserve; each query keeps up to
                         2 (k + margin) + 128 bound pairs before compacting */
  int32_t autotune;   /* batched form: pick tiles per cloud-size bucket      */
  int32_t flags;      /* KNN_SQUARED_DIST | KNN_NO_TENSOR_CORES, or 0        */
  int32_t lloyd_iters;/* representative refinement: after the draw, this many
                         steps of "move every representative to its cluster's
                         centroid, re-assign" (0 = the reference's draw only;
                         default 0)                                          */
  int32_t reserved0;
} knn_options;

/*
 * Statistics of one call (the reference prints stage timers, common8.h:83-90,
 * and the evaluation counter `Total`, knnjoin.cu:565-570, 804).
 */
typedef struct knn_stats {
  int64_t dist_evals;       /* exact query-to-point distances evaluated       */
  int64_t pairs_total;      /* m * n                                          */
  int64_t pairs_pruned;     /* pairs_total - dist_evals                       */
  int64_t clusters_visited; /* (query, reference cluster) pairs scanned        */
  int64_t clusters_pruned;  /* (query, reference cluster) pairs skipped whole  */
  int64_t fp64_rechecks;    /* candidates inside the FP32 rounding band of the
                               k-th distance whose order was re-decided in FP64
                               (both forms)                                   */
  int64_t topk_candidates;  /* candidates that beat the running k-th key       */
  int64_t topk_merges;      /* sorted merges of candidate buffers into top-k   */
  float ms_build;           /* representative sampling .. cluster filter      */
  float ms_search;          /* per-query pruned scan                          */
  float ms_total;           /* whole call, device time                        */
  int32_t qreps_used;
  int32_t sreps_used;
  int32_t kernels_launched; /* device kernels this call enqueued (a radix sort
                               counts as one)                                 */
  int32_t refine_fallbacks; /* BF16 form: queries whose kept candidates did
                               not fit the re-ranking buffer and went to the
                               FP32 scan instead                              */
  int32_t band_queries;     /* queries whose k-th boundary was settled by the
                               band kernel (a key of the band did not fit the
                               scan's candidate list)                         */
} knn_stats;

/* Fill `opt` with the defaults listed above. */
void knn_default_options(knn_options *opt);

/* Message for the last failing call on this host thread ("" if none). */
const char *knn_last_error(void);

/* ABI version (KNNSWEET_ABI_VERSION). */
int32_t knn_abi_version(void);

/*
 * Exact kNN join on host buffers.  Replaces the whole reference pipeline
 * main -> clusterReps -> RepsUpperBound -> FilterReps -> KNNQuery_base
 * (src/knnjoin.cu:983-1145): copies q (m x d) and r (n x d) to the GPU, joins,
 * and copies the m x k result back into out_idx / out_dist (host memory).
 * `opt` may be NULL (defaults); `st` may be NULL.
 */
int knn_join(const float *q, int64_t m, const float *r, int64_t n, int32_t d,
             int32_t k, int32_t *out_idx, float *out_dist,
             const knn_options *opt, knn_stats *st);

/*
 * Same join on device buffers (all four pointers are device memory of the
 * current device), enqueued on `stream` (a cudaStream_t; NULL = legacy default
 * stream).  Internal scratch comes from the stream-ordered allocator and is
 * released before return.  Returns after enqueueing unless `st` is non-NULL,
 * in which case it synchronises the stream to fill the statistics.
 * q may equal r (self-join, as in run_sample.sh:1); then m must equal n.
 */
int knn_join_device(const float *q, int64_t m, const float *r, int64_t n,
                    int32_t d, int32_t k, int32_t *out_idx, float *out_dist,
                    const knn_options *opt, knn_stats *st, void *stream);

/*
 * Gradient of a loss over kNN pairs (no reference counterpart; the reference
 * has no gradient).  For every pair (i, j=idx[i*k+t]) with upstream gradient
 * g = grad_dist2[i*k+t] on the squared distance |q_i - r_j|^2:
 *   grad_q[i] += 2 g (q_i - r_j),   grad_r[j] -= 2 g (q_i - r_j).
 * Pairs with idx < 0 are skipped.  grad_q (m x d) and grad_r (n x d) are
 * device buffers that are ACCUMULATED into (zero them first for a plain
 * gradient); grad_r may be NULL.  Device pointers, enqueued on `stream`.
 */
int knn_backward_device(const float *q, int64_t m, const float *r, int64_t n,
                        int32_t d, int32_t k, const int32_t *idx,
                        const float *grad_dist2, float *grad_q, float *grad_r,
                        void *stream);

/*
 * Allocation-free variant of knn_join_device.  It has no counterpart in the
 * reference (which cudaMallocs everything and never frees it).
 *
 * For callers that may not allocate device memory: applications that reserve
 * the whole GPU for their own memory manager at start-up, and code that must
 * not allocate once running because cudaMalloc / cudaFree can block and
 * synchronise the device.  The caller passes device inputs and outputs
 * exactly as for knn_join_device; every other buffer the join needs is carved
 * from one array of KNN_NOALLOC_SCRATCH_BYTES compiled into the library, and
 * the call makes no cudaMalloc, cudaFree or other allocating call.
 *  - Limit: a join whose scratch exceeds KNN_NOALLOC_SCRATCH_BYTES (32 MiB;
 *    about 250,000 points for a d = 3 self-join with 800 representatives) is
 *    rejected with KNN_EINVAL and a message giving the bytes it would need.
 *  - Every GPU that loads the library holds the array until the process
 *    exits.  The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture.
 *  - All calls on a device share the one array, and it keeps the previous
 *    call's contents: calls that overlap on the GPU (different streams, or
 *    host threads racing) corrupt each other.  Serialise them.
 *  - No statistics: the stats-filling path of knn_join_device creates events.
 *  - Options: qreps, sreps, seed, rep_trials, KNN_SQUARED_DIST and
 *    KNN_NO_TENSOR_CORES act as for knn_join_device; precision must be
 *    KNN_FP32 and lloyd_iters 0 (anything else is refused with KNN_EINVAL and
 *    a message naming the option).
 */
#define KNN_NOALLOC_SCRATCH_BYTES (32u << 20)
int knn_join_device_noalloc(const float *q, int64_t m, const float *r, int64_t n,
                            int32_t d, int32_t k, int32_t *out_idx,
                            float *out_dist, const knn_options *opt,
                            void *stream);

/*
 * Batched join: `ncloud` independent joins in one call (no reference
 * counterpart as an entry point; per cloud it computes what one reference
 * run, src/knnjoin.cu:983-1145, computes for one pair of point sets).
 * Cloud c's queries are rows q_offsets[c] .. q_offsets[c+1]-1 of q and its
 * reference points rows r_offsets[c] .. r_offsets[c+1]-1 of r; every query
 * gets its k nearest among its own cloud's reference points only, and
 * out_idx holds indices RELATIVE to r_offsets[c] (0-based within the cloud),
 * rows in q's order, -1 / +inf where the cloud has fewer than k points.
 *  - q, r, out_idx, out_dist: device memory; q_offsets, r_offsets: HOST
 *    arrays of ncloud + 1 non-decreasing int64 starting at 0.
 *  - Passing q == r and equal offsets makes it a per-cloud self-join.
 *  - 1 <= d <= 32, 1 <= k <= 256.  qreps / sreps / lloyd_iters / margin are
 *    ignored: each cloud of n points gets about alpha * sqrt(n)
 *    representatives (at most 2048), alpha chosen per cloud-size bucket
 *    (powers of two) by timing when opt->autotune is set (the first call per
 *    (d, k, bucket) synchronises the stream; the choice is cached for the
 *    process), 1.6 otherwise.  Representative draws use a counter-based
 *    hash of (seed, cloud, trial, slot), best of rep_trials by spread.
 *  - Once tuned, the call enqueues without host synchronisation (unless `st`
 *    is given) and its scratch comes from the library's stream-ordered pool.
 */
int knn_join_batched_device(const float *q, const int64_t *q_offsets,
                            const float *r, const int64_t *r_offsets,
                            int32_t ncloud, int32_t d, int32_t k,
                            int32_t *out_idx, float *out_dist,
                            const knn_options *opt, knn_stats *st,
                            void *stream);

/*
 * knn_join_batched_device on HOST buffers: q, r, out_idx and out_dist are host
 * memory (the reference keeps its inputs and result in host arrays,
 * src/knnjoin.cu:1003-1033, and runs one pair of point sets per process).  The
 * clouds are copied to the current device on a stream of the calling thread,
 * joined, and the result copied back; the call returns when it is complete.
 * Offsets, limits, options and results as for knn_join_batched_device.
 */
int knn_join_batched(const float *q, const int64_t *q_offsets, const float *r,
                     const int64_t *r_offsets, int32_t ncloud, int32_t d, int32_t k,
                     int32_t *out_idx, float *out_dist, const knn_options *opt,
                     knn_stats *st);

/*
 * Reusable index of a reference set.  The reference rebuilds everything on
 * every run (clusterReps, src/knnjoin.cu:166-411), although its source side --
 * representatives, assignment, sorted member lists (knnjoin.cu:223-240,
 * 331-399) -- depends only on the reference points.  knn_index_build does that
 * part once, on the current device and `stream`, keeping a copy of the points;
 * it returns when the build is complete.  Options that shape it: sreps, seed,
 * rep_trials, lloyd_iters, KNN_NO_TENSOR_CORES.
 * knn_index_query then joins any number of query batches against it: the same
 * result as knn_join_device with the same options (the query-side options:
 * qreps, precision, margin, KNN_SQUARED_DIST), device buffers, enqueued on
 * `stream`; it must run on the index's device.  Queries may run concurrently
 * on different streams (the index is read-only).  knn_index_free releases the
 * index (it synchronises); knn_index_info reports n, d and the representatives.
 */
typedef struct knn_index knn_index;
int knn_index_build(const float *r, int64_t n, int32_t d, const knn_options *opt,
                    knn_index **out, void *stream);
int knn_index_query(const knn_index *index, const float *q, int64_t m, int32_t k,
                    int32_t *out_idx, float *out_dist, const knn_options *opt,
                    knn_stats *st, void *stream);
int knn_index_free(knn_index *index);
int knn_index_info(const knn_index *index, int64_t *n, int32_t *d, int32_t *reps);

/*
 * knn_join over several GPUs of this process.  No counterpart in the
 * reference, which runs its search on one GPU (src/knnjoin.cu:1103-1129).
 * Host buffers as in knn_join.  The reference index and the query clusters
 * are built once, on devices[0]; the query clusters are split into ndev
 * contiguous ranges balanced by their estimated work (query count times the
 * band sizes they can scan), so no query cluster is split; every other listed
 * device receives a peer copy of what the search reads and searches its range,
 * storing its results into devices[0]'s result buffer through peer memory
 * (into a local buffer merged on devices[0] where peer access is missing).
 * An id may repeat: its shards then run concurrently on separate streams.
 * The result is knn_join's.  stats (optional): counts summed over the shards,
 * ms_build the build on devices[0], ms_search the slowest shard (peer copies
 * included).  Errors: the first failing call's code and message.
 */
int knn_join_sharded(const float *q, int64_t m, const float *r, int64_t n, int32_t d,
                     int32_t k, int32_t *out_idx, float *out_dist, const knn_options *opt,
                     const int32_t *devices, int32_t ndev, knn_stats *stats);

/*
 * One part of a join split across processes (one process per GPU, e.g. under
 * torchrun): every process calls it with the same inputs and options on its
 * own device and stream, part = its rank, nparts = the number of processes.
 * Each builds the same index (the build is deterministic), computes the same
 * partition of the query clusters as knn_join_sharded and searches only part
 * `part`: the result rows of those queries are written into out_idx /
 * out_dist (device, m x k; other rows are left untouched), their query row
 * ids into out_rows[0 .. *out_count) (device, room for m; may be NULL), and
 * *out_count (host) is set.  Synchronises the stream once (to plan the
 * partition).  The parts of all processes together are knn_join's result.
 * No reference counterpart.
 */
int knn_join_partition_device(const float *q, int64_t m, const float *r, int64_t n,
                              int32_t d, int32_t k, int32_t part, int32_t nparts,
                              int32_t *out_idx, float *out_dist, int32_t *out_rows,
                              int64_t *out_count, const knn_options *opt, knn_stats *st,
                              void *stream);

/*
 * Returns the device scratch memory the library keeps cached between calls
 * (one stream-ordered pool per device; no reference counterpart: the
 * reference never frees its device memory).  Memory still in use by calls in
 * flight is kept.
 */
int knn_trim_memory(void);

/*
 * Interleave SoA results into the reference's IndexDist layout
 * {int32 index; float dist} (include/common8.h:37-40), host memory,
 * `count` = m * k entries.  out must hold 2*count 32-bit words.
 */
void knn_pack_indexdist(const int32_t *idx, const float *dist, int64_t count,
                        void *out);

#ifdef __cplusplus
}
#endif

#endif /* KNNSWEET_H */
