// api.cu -- orchestration of the exact kNN join and the C ABI entry points.
//
// Pipeline of one join (knn_join_device), all on one stream, no host round
// trips after the representative draw:
//   reference side: pack rows -> draw representatives (10 seeded trials,
//     best spread) -> nearest representative per point -> one radix sort by
//     (cluster, distance to representative) -> cluster-contiguous rows,
//     member distances, offsets, min/max member distance
//   query side: the same (shared with the reference side for a self-join)
//   bounds: rep-rep distances -> per query cluster k-th upper bound and the
//     surviving reference clusters, nearest first
//   scan: one warp per query over its surviving clusters (scan.cu)
// The reference runs the same stages with host sorts and per-cluster
// device<->host copies in between (src/knnjoin.cu:166-411, 1043-1133).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "glibc_rand.h"

// A host-buffer join's first copy-back chunk holds one query per resident
// scan warp (1), or all chunks are equal (0).
#ifndef KNN_SMALL_FIRST_CHUNK
#define KNN_SMALL_FIRST_CHUNK 1
#endif
#include "kernels.cuh"
#include "pipeline.cuh"

namespace knnsweet {

std::string &error_buffer() {
  thread_local std::string s;
  return s;
}

int &launch_counter() {
  thread_local int n = 0;
  return n;
}

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  error_buffer() = buf;
}

// One stream-ordered memory pool per device for the library's scratch.  Its
// release threshold is unlimited, so memory freed at the end of a call stays
// cached for the next call instead of going back to the driver at every
// synchronisation (knn_trim_memory() returns it).
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};

int scratch_pool(cudaMemPool_t *out) {
  int dev = 0;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d out of range", dev);
    return KNN_EINVAL;
  }
  std::lock_guard<std::mutex> guard(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    KNN_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    KNN_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return KNN_OK;
}

// Argument ranges shared by every entry point.
int check_sizes(int64_t m, int64_t n, int32_t d, int32_t k) {
  if (d <= 0) {
    set_error("d must be positive (got %d)", d);
    return KNN_EINVAL;
  }
  if (k <= 0 || k > KNN_MAX_K) {
    set_error("k must be in [1, %d] (got %d)", KNN_MAX_K, k);
    return KNN_EINVAL;
  }
  if (m < 0 || n < 0 || m > INT32_MAX || n > INT32_MAX) {
    set_error("m and n must be in [0, 2^31-1]");
    return KNN_EINVAL;
  }
  if (n > 0 && (int64_t)d > ((int64_t)1 << 40) / n) {
    set_error("n * d too large");
    return KNN_EINVAL;
  }
  return KNN_OK;
}

// Option ranges shared by every entry point.
int check_options(const knn_options *opt, knn_options *o) {
  knn_default_options(o);
  if (opt) *o = *opt;
  if (o->qreps < 0 || o->sreps < 0 || o->qreps > KNN_MAX_REPS ||
      o->sreps > KNN_MAX_REPS) {
    set_error("qreps/sreps must be in [0, %d]", KNN_MAX_REPS);
    return KNN_EINVAL;
  }
  if (o->rep_trials <= 0 || o->rep_trials > 1000) {
    set_error("rep_trials must be in [1, 1000]");
    return KNN_EINVAL;
  }
  if (o->precision != KNN_FP32 && o->precision != KNN_BF16_REFINE) {
    set_error("unknown precision %d", o->precision);
    return KNN_EINVAL;
  }
  if (o->margin < 0 || o->margin > 4096) {
    set_error("margin must be in [0, 4096]");
    return KNN_EINVAL;
  }
  if (o->lloyd_iters < 0 || o->lloyd_iters > 100) {
    set_error("lloyd_iters must be in [0, 100]");
    return KNN_EINVAL;
  }
  if ((o->flags & ~(KNN_SQUARED_DIST | KNN_NO_TENSOR_CORES)) != 0) {
    set_error("unknown flags 0x%x", o->flags);
    return KNN_EINVAL;
  }
  return KNN_OK;
}



__global__ void fill_empty_kernel(int32_t *idx, float *dist, int64_t count) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    idx[t] = -1;
    dist[t] = __int_as_float(0x7f800000);
  }
}

// Small host arrays reach the device as kernel parameters (up to 8,000
// words per launch): a pageable cudaMemcpyAsync would wait for the stream to
// drain first, stalling back-to-back joins at every call.
struct ParamChunk {
  int32_t count;
  int32_t v[8000];
};

__global__ void upload_kernel(int32_t *__restrict__ dst, const ParamChunk c) {
  for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[i] = c.v[i];
}

int upload_i32(const std::vector<int32_t> &src, int32_t *dst, cudaStream_t s) {
  ParamChunk c;
  for (size_t base = 0; base < src.size(); base += 8000) {
    size_t cnt = std::min<size_t>(8000, src.size() - base);
    c.count = (int32_t)cnt;
    memcpy(c.v, src.data() + base, cnt * sizeof(int32_t));
    upload_kernel<<<1, 256, 0, s>>>(dst + base, c);
    KNN_LAUNCH_CHECK();
  }
  return KNN_OK;
}

// Representative count when the caller passes 0: about 1.6 sqrt(n)
// (the reference's sample run uses 800 for 145,057 points, run_sample.sh:1).
int default_reps(int64_t n) {
  double r = std::floor(1.6 * std::sqrt((double)n) + 0.5);
  if (r < 1) r = 1;
  if (r > 4096) r = 4096;
  return (int)r;
}


int build_clusters(Arena &keep, Arena &ar, const float4 *rows, int64_t n, int d, int dp4s, int R,
                   uint32_t seed, int trials, int lloyd_iters, bool use_tc, int *err,
                   cudaStream_t s, ClusterSet *cs) {
  cs->R = R;
  // representative draw on the host: trials x R indices rand() % n
  std::vector<int32_t> cand((size_t)trials * R);
  GlibcRand g(seed);
  for (auto &c : cand) c = g.next() % (int32_t)n;
  int32_t *cand_dev;
  uint32_t *score;
  KNN_TRY(ar.alloc(&cand_dev, cand.size()));
  KNN_TRY(ar.alloc(&score, (size_t)trials));
  KNN_TRY(upload_i32(cand, cand_dev, s));
  KNN_TRY(keep.alloc(&cs->reps, (size_t)R * dp4s));
  KNN_TRY(keep.alloc(&cs->rep_rows, (size_t)R));
  KNN_TRY(launch_rep_select(rows, dp4s, cand_dev, R, trials, score, cs->reps,
                            cs->rep_rows, s));
  int32_t *cl;
  float *dr;
  KNN_TRY(ar.alloc(&cl, (size_t)n));
  KNN_TRY(ar.alloc(&dr, (size_t)n));
  const bool tc_assign = use_tc && assign_tc_supported(d);
  unsigned char *tc_scratch = nullptr;
  if (tc_assign) KNN_TRY(ar.alloc(&tc_scratch, assign_tc_scratch_bytes(R, d)));
  uint64_t *keys;
  int32_t *vals;
  KNN_TRY(ar.alloc(&keys, (size_t)n));
  KNN_TRY(ar.alloc(&vals, (size_t)n));
  KNN_TRY(keep.alloc(&cs->skeys, (size_t)n));
  KNN_TRY(keep.alloc(&cs->perm, (size_t)n));
  size_t temp_bytes = cluster_sort_temp_bytes(n, R);
  unsigned char *temp;
  KNN_TRY(ar.alloc(&temp, temp_bytes));
  KNN_TRY(keep.alloc(&cs->off, (size_t)R + 1));
  // nearest representative (BF16 tensor-core arg-min + exact FP32 distance to
  // the winner for d >= 16, FP32 CUDA cores otherwise), then one sort into
  // clusters; with Lloyd steps the representatives move to their clusters'
  // centroids (the smallest clusters' representatives to the farthest member
  // of the widest clusters) and the points are assigned and sorted again
  for (int it = 0; it <= lloyd_iters; it++) {
    if (it > 0) {
      KNN_TRY(launch_centroids(rows, dp4s, cs->perm, cs->off, R, cs->reps, s));
      KNN_TRY(launch_split_clusters(rows, dp4s, cs->perm, cs->off, cs->skeys, R, cs->reps, s));
    }
    if (tc_assign)
      KNN_TRY(launch_assign_tc(rows, n, dp4s, d, cs->reps, R, tc_scratch, cl, dr, err, s));
    else
      KNN_TRY(launch_assign(rows, n, dp4s, cs->reps, R, cl, dr, s));
    KNN_TRY(launch_cluster_sort(cl, dr, n, R, keys, vals, cs->skeys, cs->perm, temp,
                                temp_bytes, s));
    KNN_TRY(launch_cluster_offsets(cs->skeys, n, R, cs->off, s));
  }
  return KNN_OK;
}



struct EventSet {
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  bool on = false;
  ~EventSet() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
  int create() {
    for (auto &e : ev) KNN_CUDA_TRY(cudaEventCreate(&e));
    on = true;
    return KNN_OK;
  }
  int record(int i, cudaStream_t s) {
    if (on) KNN_CUDA_TRY(cudaEventRecord(ev[i], s));
    return KNN_OK;
  }
};


// Events of the chunked copies, destroyed once both streams are idle.
// Events of the chunked copies: the calling thread's, created on first use
// and reused (a call leaves its streams idle, so the previous call's events
// have completed).
int chunk_events(int n, std::vector<cudaEvent_t> **out) {
  thread_local std::vector<cudaEvent_t> pool;
  while ((int)pool.size() < n) {
    cudaEvent_t e;
    KNN_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    pool.push_back(e);
  }
  *out = &pool;
  return KNN_OK;
}

// Row geometry: float4 chunks per row (rounded up to a power of two for the
// register-width scan kernels when d <= 32) and the scan template width.
void row_geometry(int d, int *dp4s, int *tmpl) {
  const int dp4 = (d + 3) / 4;
  *dp4s = dp4;
  *tmpl = 0;
  if (dp4 <= 8) {
    int p = 1;
    while (p < dp4) p <<= 1;
    *dp4s = p;
    *tmpl = p;
  }
}


// Builds the reference side; the arrays it keeps come from `keep`, scratch
// from `tmp`.  With copy_rows the packed rows are always a copy (an index
// must not depend on the caller's buffer).
int build_ref_side(Arena &keep, Arena &tmp, const float *r, int64_t n, int d, int Rs,
                   const knn_options &o, bool copy_rows, int *dev_err, cudaStream_t s,
                   RefSide *R) {
  R->n = n;
  R->d = d;
  row_geometry(d, &R->dp4s, &R->tmpl);
  R->Rs = Rs;
  const int dp4s = R->dp4s;
  if (!copy_rows && dp4s * 4 == d && (reinterpret_cast<uintptr_t>(r) & 15) == 0) {
    R->Rp = reinterpret_cast<const float4 *>(r);
  } else {
    float4 *p;
    KNN_TRY(keep.alloc(&p, (size_t)n * dp4s));
    KNN_TRY(launch_pack_rows(r, n, d, dp4s, p, s));
    R->Rp = p;
  }
  KNN_TRY(keep.alloc(&R->inexact, 1));
  KNN_CUDA_TRY(cudaMemsetAsync(R->inexact, 0, sizeof(int), s));
  KNN_TRY(launch_exact_check(reinterpret_cast<const float *>(R->Rp), n * dp4s * 4, d,
                             R->inexact, s));
  const bool use_tc = (o.flags & KNN_NO_TENSOR_CORES) == 0;
  KNN_TRY(build_clusters(keep, tmp, R->Rp, n, d, dp4s, Rs, o.seed, o.rep_trials, o.lloyd_iters,
                         use_tc, dev_err, s, &R->sset));
  KNN_TRY(keep.alloc(&R->srows, (size_t)n * dp4s));
  KNN_TRY(keep.alloc(&R->sdist, (size_t)n));
  KNN_TRY(keep.alloc(&R->sidx, (size_t)n));
  KNN_TRY(keep.alloc(&R->cmin, (size_t)Rs));
  KNN_TRY(keep.alloc(&R->cmax, (size_t)Rs));
  // rows with a spare pad float carry their index there (register-width rows)
  R->idx_in_row = R->tmpl > 0 && 4 * dp4s > d;
  KNN_TRY(launch_cluster_layout(R->sset.skeys, R->sset.perm, n, R->Rp, dp4s, R->idx_in_row,
                                R->srows, R->sdist, R->sidx, s));
  KNN_TRY(launch_cluster_minmax(R->sset.off, R->sdist, Rs, R->cmin, R->cmax, s));
  return KNN_OK;
}

// Number of query representatives for m queries (self: the join shares the
// reference clusters when the counts agree).
int query_rep_count(const knn_options &o, int64_t m, int d, int k, bool self, int Rs) {
  int Rq = o.qreps > 0 ? o.qreps : (self ? Rs : default_reps(m));
  // the tensor-core tiles hold 128 queries of one query cluster: by default
  // the BF16 form sizes the query clusters to fill them
  if (o.qreps <= 0 && !self && o.precision == KNN_BF16_REFINE && tile_search_supported(d, k, o.margin))
    Rq = (int)std::min<int64_t>(KNN_MAX_REPS, std::max<int64_t>(1, (m + 127) / 128));
  if (Rq > m) Rq = (int)m;
  return Rq;
}

int query_impl(const RefSide &R, bool share, const float *q, int64_t m, int32_t k,
               int32_t *out_idx, float *out_dist, const knn_options &o, knn_stats *st,
               cudaStream_t s, HostSink *sink, Arena &ar, EventSet &evs,
               unsigned long long *ctr);

int join_device_impl(const float *q, int64_t m, const float *r, int64_t n,
                     int32_t d, int32_t k, int32_t *out_idx, float *out_dist,
                     const knn_options *opt, knn_stats *st, cudaStream_t s,
                     HostSink *sink = nullptr) {
  knn_options o;
  KNN_TRY(check_options(opt, &o));
  KNN_TRY(check_sizes(m, n, d, k));
  if (st) memset(st, 0, sizeof *st);
  launch_counter() = 0;
  if (m == 0) return KNN_OK;
  if (!q || (!r && n > 0) || !out_idx || !out_dist) {
    set_error("null pointer argument");
    return KNN_EINVAL;
  }
  if (st) st->pairs_total = m * n;
  if (n == 0) {
    fill_empty_kernel<<<256, 256, 0, s>>>(out_idx, out_dist, m * (int64_t)k);
    KNN_LAUNCH_CHECK();
    return KNN_OK;
  }
  const bool self = (q == r) && (m == n);
  int Rs = o.sreps > 0 ? o.sreps : default_reps(n);
  if (Rs > n) Rs = (int)n;
  const int Rq = query_rep_count(o, m, d, k, self, Rs);
  const bool share = self && Rq == Rs;

  EventSet evs;
  if (st) KNN_TRY(evs.create());
  KNN_TRY(evs.record(0, s));
  Arena ar(s);
  unsigned long long *ctr;
  KNN_TRY(ar.alloc(&ctr, kCtrCount));
  KNN_CUDA_TRY(cudaMemsetAsync(ctr, 0, kCtrCount * sizeof(unsigned long long), s));
  RefSide R;
  KNN_TRY(build_ref_side(ar, ar, r, n, d, Rs, o, false, reinterpret_cast<int *>(ctr + kCtrErr),
                         s, &R));
  return query_impl(R, share, q, m, k, out_idx, out_dist, o, st, s, sink, ar, evs, ctr);
}


int build_query_side(const RefSide &R, bool share, const float *q, int64_t m, int32_t k,
                     const knn_options &o, Arena &ar, unsigned long long *ctr, cudaStream_t s,
                     QuerySide *Q) {
  const int d = R.d, dp4s = R.dp4s, Rs = R.Rs;
  const int Rq = share ? Rs : query_rep_count(o, m, d, k, false, Rs);
  int *dev_err = reinterpret_cast<int *>(ctr + kCtrErr);
  const bool use_tc = (o.flags & KNN_NO_TENSOR_CORES) == 0;
  Q->Rq = Rq;
  Q->inexact = R.inexact;
  if (share) {
    Q->Qp = R.Rp;
    Q->qset = R.sset;
  } else {
    if (dp4s * 4 == d && (reinterpret_cast<uintptr_t>(q) & 15) == 0) {
      Q->Qp = reinterpret_cast<const float4 *>(q);
    } else {
      float4 *p;
      KNN_TRY(ar.alloc(&p, (size_t)m * dp4s));
      KNN_TRY(launch_pack_rows(q, m, d, dp4s, p, s));
      Q->Qp = p;
    }
    int *qf = reinterpret_cast<int *>(ctr + kCtrInexactQ);
    KNN_TRY(launch_exact_check(reinterpret_cast<const float *>(Q->Qp), m * dp4s * 4, d, qf, s));
    Q->inexact = qf;
    KNN_TRY(build_clusters(ar, ar, Q->Qp, m, d, dp4s, Rq, o.seed, o.rep_trials, o.lloyd_iters,
                           use_tc, dev_err, s, &Q->qset));
  }
  KNN_TRY(ar.alloc(&Q->qrad, (size_t)Rq));
  KNN_TRY(ar.alloc(&Q->slot_cl, (size_t)m));
  KNN_TRY(launch_query_clusters(Q->qset.skeys, Q->qset.off, m, Rq, Q->qrad, Q->slot_cl, s));
  KNN_TRY(ar.alloc(&Q->drr, (size_t)Rq * Rs));
  KNN_TRY(launch_rep_dist(Q->qset.reps, Rq, R.sset.reps, Rs, dp4s, Q->drr, s));
  KNN_TRY(ar.alloc(&Q->theta0, (size_t)Rq));
  KNN_TRY(ar.alloc(&Q->rlist, (size_t)Rq * Rs));
  KNN_TRY(ar.alloc(&Q->rlen, (size_t)Rq));
  KNN_TRY(ar.alloc(&Q->clb, (size_t)Rq * ((Rs + 31) / 32)));
  KNN_TRY(launch_bounds_filter(Q->drr, Rq, Rs, Q->qrad, Q->qset.off, R.sset.off, R.sdist, R.cmax,
                               k, d, Q->theta0, Q->rlist, Q->rlen, Q->clb, s));
  return KNN_OK;
}

// The search of the query clusters c0 .. c1-1, whose slots are
// slot0 .. slot0+nslot-1: the BF16 tile search (precision BF16_REFINE) and
// the FP32 scan, results into rows of out_idx / out_dist (query order).
// `ctr` (kCtrCount counters, zeroed) on the searching device.  With a host
// sink and the whole query set, the scan runs in row chunks whose results
// are copied back while the next chunk runs.
int search_clusters(const RefSide &R, const QuerySide &Q, int64_t m, int32_t k, int c0, int c1,
                    int64_t slot0, int64_t nslot, int32_t *out_idx, float *out_dist,
                    const knn_options &o, cudaStream_t s, HostSink *sink, Arena &ar,
                    unsigned long long *ctr) {
  if (nslot == 0) return KNN_OK;
  const int d = R.d, dp4s = R.dp4s, Rs = R.Rs;
  int dev = 0, num_sms = 148;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  KNN_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  const int nclu = c1 - c0;

  // BF16+refine form: tensor-core tiles over the same candidate lists; the
  // FP32 scan below then runs only for the queries the tiles hand back.
  int grid = 0, cap = 0, P = 0;
  size_t smem = 0;
  const bool tiles = o.precision == KNN_BF16_REFINE && tile_search_supported(d, k, o.margin) &&
                     tile_search_geometry(d, k, o.margin, num_sms, &grid, &cap, &P, &smem) ==
                         KNN_OK;
  int32_t *fb_slots = nullptr;
  unsigned *fb_count = reinterpret_cast<unsigned *>(ctr + kCtrFallback);
  if (tiles) {
    grid = (int)std::min<int64_t>(grid, nslot / 128 + nclu + 1);
    int32_t *tile_list, *ntiles;
    float2 *buf_lu;
    int32_t *buf_pos;
    const size_t slots = (size_t)grid * 128 * cap;
    KNN_TRY(ar.alloc(&tile_list, (size_t)4 * (nslot / 128 + nclu + 1)));
    KNN_TRY(ar.alloc(&ntiles, 1));
    KNN_TRY(ar.alloc(&buf_lu, slots));
    KNN_TRY(ar.alloc(&buf_pos, slots));
    KNN_TRY(ar.alloc(&fb_slots, (size_t)nslot));
    KNN_TRY(launch_tile_list(Q.qset.off + c0, nclu, c0, tile_list, ntiles, s));
    TileArgs t{};
    t.qrows = Q.Qp;
    t.dp4 = dp4s;
    t.d = d;
    t.KD = 16;
    while (t.KD < d) t.KD <<= 1;
    t.qorder = Q.qset.perm;
    t.tiles = tile_list;
    t.ntiles = ntiles;
    t.srows = R.srows;
    t.sidx = R.sidx;
    t.rrows = R.Rp;
    t.soff = R.sset.off;
    t.sdist = R.sdist;
    t.cmin = R.cmin;
    t.cmax = R.cmax;
    t.sreps = R.sset.reps;
    t.rlist = Q.rlist;
    t.rlen = Q.rlen;
    t.Rs = Rs;
    t.clb = Q.clb;
    t.clb_stride = (Rs + 31) / 32;
    t.qkeys = Q.qset.skeys;
    t.theta0 = Q.theta0;
    t.k = k;
    t.cap = cap;
    t.P = P;
    t.squared = (o.flags & KNN_SQUARED_DIST) != 0;
    t.buf_lu = buf_lu;
    t.buf_pos = buf_pos;
    t.out_idx = out_idx;
    t.out_dist = out_dist;
    t.work = ctr + kCtrTileWork;
    t.fb_slots = fb_slots;
    t.fb_count = fb_count;
    t.err = reinterpret_cast<int *>(ctr + kCtrErr);
    t.counters = ctr + kCtrTile;
    KNN_TRY(launch_tile_search(t, grid, smem, s));
  }

  ScanArgs a{};
  a.qrows = Q.Qp;
  a.qorder = Q.qset.perm;
  a.slot_cl = Q.slot_cl;
  a.m = nslot;
  a.slot_base = slot0;
  a.d = d;
  a.dp4 = dp4s;
  a.dp4_tmpl = R.tmpl;
  a.k = k;
  a.idx_in_row = R.idx_in_row;
  a.squared = (o.flags & KNN_SQUARED_DIST) != 0;
  a.sreps = R.sset.reps;
  a.srows = R.srows;
  a.sdist = R.sdist;
  a.sidx = R.sidx;
  a.soff = R.sset.off;
  a.cmin = R.cmin;
  a.cmax = R.cmax;
  a.theta0 = Q.theta0;
  a.qrad = Q.qrad;
  a.qkeys = Q.qset.skeys;
  a.rlist = Q.rlist;
  a.rlen = Q.rlen;
  a.clb = Q.clb;
  a.clb_stride = (Rs + 31) / 32;
  a.Rs = Rs;
  a.n_ref = R.n;
  a.rrows = R.Rp;
  a.inexact_r = R.inexact;
  a.inexact_q = Q.inexact;
  a.out_idx = out_idx;
  a.out_dist = out_dist;
  KNN_TRY(ar.alloc(&a.unres_slot, (size_t)nslot));
  a.unres_count = reinterpret_cast<unsigned *>(ctr + kCtrUnres);
  a.work_counter = ctr + kCtrWork;
  a.counters = ctr + kCtrScan;
  if (tiles) {
    a.slot_list = fb_slots;
    a.slot_count = fb_count;
  }
  // host destination and a large result: scan in row chunks (each chunk's
  // slots still in query-cluster order) and copy every finished chunk back
  // while the next one runs.  About 16 MB of results per chunk, 8 to 32
  // chunks (k = 200 self-join, 392 MB of results: 8.43 ms end to end with 8
  // chunks, 8.18 with 24, 8.17 with 32; the copy alone takes 6.89 ms), the
  // first one small (8.23 -> 8.10 ms on a box whose copy takes 7.15 ms)
  const int64_t out_bytes = m * (int64_t)k * 8;
  const bool whole = slot0 == 0 && nslot == m;
  const int nchunks =
      (sink && whole && !tiles && out_bytes >= (16 << 20) && m >= 8 * 1024)
          ? (int)std::min<int64_t>(32, std::max<int64_t>(8, out_bytes >> 24))
          : 1;
  if (nchunks > 1) {
    // the first chunk one query per resident warp of the scan, so that the
    // copy-back starts after about one query's time; the rest in equal chunks
    const int64_t first =
        KNN_SMALL_FIRST_CHUNK ? std::min<int64_t>(m / 4, (int64_t)num_sms * 32) : 0;
    const int nrest = first > 0 ? nchunks - 1 : nchunks;
    const int chunk_rows = (int)((m - first + nrest - 1) / nrest);
    std::vector<int64_t> r0s(nchunks);
    std::vector<int32_t> counts(nchunks);
    for (int c = 0; c < nchunks; c++) {
      const int64_t b = first > 0 ? (c == 0 ? 0 : first + (int64_t)(c - 1) * chunk_rows)
                                  : (int64_t)c * chunk_rows;
      const int64_t e = first > 0 && c == 0 ? first : std::min<int64_t>(m, b + chunk_rows);
      r0s[c] = std::min<int64_t>(b, m);
      counts[c] = (int32_t)std::max<int64_t>(0, e - r0s[c]);
    }
    uint32_t *ckeys, *ckeys_out;
    int32_t *cvals, *cslots, *ccount;
    unsigned long long *cwork;
    const size_t tb = chunk_slots_temp_bytes(m, nchunks);
    unsigned char *ctemp;
    KNN_TRY(ar.alloc(&ckeys, (size_t)m));
    KNN_TRY(ar.alloc(&ckeys_out, (size_t)m));
    KNN_TRY(ar.alloc(&cvals, (size_t)m));
    KNN_TRY(ar.alloc(&cslots, (size_t)m));
    KNN_TRY(ar.alloc(&ctemp, tb));
    KNN_TRY(ar.alloc(&ccount, (size_t)nchunks));
    KNN_TRY(ar.alloc(&cwork, (size_t)nchunks));
    KNN_CUDA_TRY(cudaMemsetAsync(cwork, 0, nchunks * sizeof(unsigned long long), s));
    KNN_TRY(upload_i32(counts, ccount, s));
    KNN_TRY(launch_chunk_slots(Q.qset.perm, m, (int)first, chunk_rows, nchunks, ckeys, ckeys_out,
                               cvals, cslots, ctemp, tb, s));
    std::vector<cudaEvent_t> *evs;
    KNN_TRY(chunk_events(nchunks, &evs));
    for (int c = 0; c < nchunks; c++) {
      if (counts[c] == 0) continue;
      const int64_t r0 = r0s[c];
      ScanArgs ac = a;
      ac.slot_list = cslots + r0;
      ac.slot_count = reinterpret_cast<const unsigned *>(ccount + c);
      ac.m = counts[c];
      ac.work_counter = cwork + c;
      KNN_TRY(launch_scan(ac, num_sms, s));
      KNN_CUDA_TRY(cudaEventRecord((*evs)[c], s));
      KNN_CUDA_TRY(cudaStreamWaitEvent(sink->copy, (*evs)[c], 0));
      const size_t cnt = (size_t)counts[c] * k;
      KNN_CUDA_TRY(cudaMemcpyAsync(sink->idx + r0 * k, out_idx + r0 * k, cnt * sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, sink->copy));
      KNN_CUDA_TRY(cudaMemcpyAsync(sink->dist + r0 * k, out_dist + r0 * k, cnt * sizeof(float),
                                   cudaMemcpyDeviceToHost, sink->copy));
    }
    sink->done = true;
  } else {
    KNN_TRY(launch_scan(a, num_sms, s));
  }
  return KNN_OK;
}

// Two non-blocking streams of the calling thread on the current device for a
// host-buffer call (the work and the copy-back), created on first use and
// kept for the thread's lifetime: creating and destroying them took about a
// quarter of a millisecond of every call.  Every host-buffer call leaves both
// idle when it returns.
int host_streams(cudaStream_t *s, cudaStream_t *cs) {
  int dev = 0;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  struct Pair {
    int dev;
    cudaStream_t s, cs;
  };
  thread_local std::vector<Pair> cache;
  for (const Pair &p : cache)
    if (p.dev == dev) {
      *s = p.s;
      *cs = p.cs;
      return KNN_OK;
    }
  Pair p{dev, nullptr, nullptr};
  KNN_CUDA_TRY(cudaStreamCreateWithFlags(&p.s, cudaStreamNonBlocking));
  if (cudaStreamCreateWithFlags(&p.cs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(p.s);
    set_error("stream creation failed");
    return KNN_ECUDA;
  }
  cache.push_back(p);
  *s = p.s;
  *cs = p.cs;
  return KNN_OK;
}

// Copies the device counters of one call into `st` (synchronises `s`).
int read_stats(const unsigned long long *ctr, cudaStream_t s, knn_stats *st) {
  unsigned long long h[kCtrCount];
  KNN_CUDA_TRY(cudaMemcpyAsync(h, ctr, sizeof h, cudaMemcpyDeviceToHost, s));
  KNN_CUDA_TRY(cudaStreamSynchronize(s));
  if (static_cast<int>(h[kCtrErr] & 0xffffffffu) != 0) {
    set_error("a bounded device wait gave up (tensor-core pipeline)");
    return KNN_ETIMEOUT;
  }
  const unsigned long long *sc = h + kCtrScan, *tc = h + kCtrTile;
  st->dist_evals += (int64_t)(sc[0] + tc[0] + tc[1]);
  st->fp64_rechecks += (int64_t)(sc[5] + tc[2]);
  st->refine_fallbacks += (int32_t)tc[3];
  st->band_queries += (int32_t)sc[6];
  st->clusters_visited += (int64_t)sc[1];
  st->clusters_pruned += (int64_t)sc[2];
  st->topk_candidates += (int64_t)sc[3];
  st->topk_merges += (int64_t)sc[4];
  return KNN_OK;
}

// The query side of a join against a built reference side.  `ctr`
// (kCtrCount counters, zeroed) and the events come from the caller; event 0
// is recorded.
int query_impl(const RefSide &R, bool share, const float *q, int64_t m, int32_t k,
               int32_t *out_idx, float *out_dist, const knn_options &o, knn_stats *st,
               cudaStream_t s, HostSink *sink, Arena &ar, EventSet &evs,
               unsigned long long *ctr) {
  if (st) st->pairs_total = m * R.n;
  QuerySide Q;
  KNN_TRY(build_query_side(R, share, q, m, k, o, ar, ctr, s, &Q));
  KNN_TRY(evs.record(1, s));
  KNN_TRY(search_clusters(R, Q, m, k, 0, Q.Rq, 0, m, out_idx, out_dist, o, s, sink, ar, ctr));
  KNN_TRY(evs.record(2, s));
  if (st) {
    KNN_TRY(read_stats(ctr, s, st));
    if (sink && sink->done) KNN_CUDA_TRY(cudaStreamSynchronize(sink->copy));
    st->pairs_pruned = st->pairs_total - st->dist_evals;
    st->qreps_used = Q.Rq;
    st->sreps_used = R.Rs;
    st->kernels_launched = launch_counter();
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_build, evs.ev[0], evs.ev[1]));
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_search, evs.ev[1], evs.ev[2]));
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_total, evs.ev[0], evs.ev[2]));
  }
  return KNN_OK;
}

// Index build / query (the reusable reference side).
int index_build_impl(const float *r, int64_t n, int32_t d, const knn_options &o,
                     cudaStream_t s, RefSide *R, std::vector<void *> *mem) {
  int Rs = o.sreps > 0 ? o.sreps : default_reps(n);
  if (Rs > n) Rs = (int)n;
  Arena keep(s);
  int rc = KNN_OK;
  {
    Arena tmp(s);
    int *err = nullptr;
    rc = tmp.alloc(&err, 1);
    if (rc == KNN_OK && cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) {
      set_error("cudaMemsetAsync failed");
      rc = KNN_ECUDA;
    }
    if (rc == KNN_OK) rc = build_ref_side(keep, tmp, r, n, d, Rs, o, true, err, s, R);
    int h = 0;
    if (rc == KNN_OK && (cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, s) !=
                             cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess)) {
      set_error("index build failed on the device: %s", cudaGetErrorString(cudaGetLastError()));
      rc = KNN_ECUDA;
    }
    if (rc == KNN_OK && h != 0) {
      set_error("a bounded device wait gave up (tensor-core pipeline)");
      rc = KNN_ETIMEOUT;
    }
  }
  if (rc == KNN_OK) *mem = keep.take();
  return rc;
}

}  // namespace knnsweet

using namespace knnsweet;

// Opaque index: the reference side of the join, kept on one device.
struct knn_index {
  int device = 0;
  RefSide *ref = nullptr;
  std::vector<void *> mem;
};

extern "C" {

int knn_index_build(const float *r, int64_t n, int32_t d, const knn_options *opt,
                    knn_index **out, void *stream) {
  error_buffer().clear();
  launch_counter() = 0;
  if (!out) {
    set_error("null index pointer");
    return KNN_EINVAL;
  }
  *out = nullptr;
  knn_options o;
  KNN_TRY(check_options(opt, &o));
  KNN_TRY(check_sizes(1, n, d, 1));
  if (n <= 0 || !r) {
    set_error("an index needs n >= 1 reference points and a device pointer");
    return KNN_EINVAL;
  }
  auto *idx = new (std::nothrow) knn_index;
  auto *R = new (std::nothrow) RefSide;
  if (!idx || !R) {
    delete idx;
    delete R;
    set_error("host allocation failed");
    return KNN_ENOMEM;
  }
  KNN_CUDA_TRY(cudaGetDevice(&idx->device));
  const int rc = index_build_impl(r, n, d, o, static_cast<cudaStream_t>(stream), R, &idx->mem);
  if (rc != KNN_OK) {
    delete R;
    delete idx;
    return rc;
  }
  idx->ref = R;
  *out = idx;
  return KNN_OK;
}

int knn_index_query(const knn_index *index, const float *q, int64_t m, int32_t k,
                    int32_t *out_idx, float *out_dist, const knn_options *opt, knn_stats *st,
                    void *stream) {
  error_buffer().clear();
  if (st) memset(st, 0, sizeof *st);
  launch_counter() = 0;
  if (!index || !index->ref) {
    set_error("null index");
    return KNN_EINVAL;
  }
  knn_options o;
  KNN_TRY(check_options(opt, &o));
  KNN_TRY(check_sizes(m, index->ref->n, index->ref->d, k));
  if (m == 0) return KNN_OK;
  if (!q || !out_idx || !out_dist) {
    set_error("null pointer argument");
    return KNN_EINVAL;
  }
  int dev = 0;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != index->device) {
    set_error("the index lives on device %d, the current device is %d", index->device, dev);
    return KNN_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  EventSet evs;
  if (st) KNN_TRY(evs.create());
  KNN_TRY(evs.record(0, s));
  Arena ar(s);
  unsigned long long *ctr;
  KNN_TRY(ar.alloc(&ctr, kCtrCount));
  KNN_CUDA_TRY(cudaMemsetAsync(ctr, 0, kCtrCount * sizeof(unsigned long long), s));
  return query_impl(*index->ref, false, q, m, k, out_idx, out_dist, o, st, s, nullptr, ar, evs,
                    ctr);
}

int knn_index_free(knn_index *index) {
  if (!index) return KNN_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(index->device);
  int rc = KNN_OK;
  for (void *p : index->mem)
    if (cudaFree(p) != cudaSuccess) rc = KNN_ECUDA;
  cudaSetDevice(prev);
  delete index->ref;
  delete index;
  if (rc != KNN_OK) set_error("cudaFree failed while releasing an index");
  return rc;
}

int knn_index_info(const knn_index *index, int64_t *n, int32_t *d, int32_t *reps) {
  if (!index || !index->ref) {
    set_error("null index");
    return KNN_EINVAL;
  }
  if (n) *n = index->ref->n;
  if (d) *d = index->ref->d;
  if (reps) *reps = index->ref->Rs;
  return KNN_OK;
}

void knn_default_options(knn_options *opt) {
  if (!opt) return;
  memset(opt, 0, sizeof *opt);
  opt->qreps = 0;
  opt->sreps = 0;
  opt->seed = 2015;
  opt->rep_trials = 10;
  opt->precision = KNN_FP32;
  opt->margin = 32;
  opt->autotune = 1;
  opt->flags = 0;
}

const char *knn_last_error(void) { return error_buffer().c_str(); }

int32_t knn_abi_version(void) { return KNNSWEET_ABI_VERSION; }

int knn_join_device(const float *q, int64_t m, const float *r, int64_t n,
                    int32_t d, int32_t k, int32_t *out_idx, float *out_dist,
                    const knn_options *opt, knn_stats *st, void *stream) {
  error_buffer().clear();
  return join_device_impl(q, m, r, n, d, k, out_idx, out_dist, opt, st,
                          static_cast<cudaStream_t>(stream));
}

int knn_join(const float *q, int64_t m, const float *r, int64_t n, int32_t d,
             int32_t k, int32_t *out_idx, float *out_dist,
             const knn_options *opt, knn_stats *st) {
  error_buffer().clear();
  {
    knn_options o;
    int rc = check_options(opt, &o);
    if (rc != KNN_OK) return rc;
    rc = check_sizes(m, n, d, k);
    if (rc != KNN_OK) return rc;
  }
  if (m == 0) {
    if (st) memset(st, 0, sizeof *st);
    return KNN_OK;
  }
  if (!q || (!r && n > 0) || !out_idx || !out_dist) {
    set_error("null pointer argument");
    return KNN_EINVAL;
  }
  cudaStream_t s, cs;
  {
    const int rc = host_streams(&s, &cs);
    if (rc != KNN_OK) return rc;
  }
  int rc = KNN_OK;
  HostSink sink{out_idx, out_dist, cs, false};
  {
    Arena ar(s);
    const bool self = (q == r) && (m == n);
    float *dq = nullptr, *dr = nullptr, *dd = nullptr;
    int32_t *di = nullptr;
    rc = ar.alloc(&dq, (size_t)m * d);
    if (rc == KNN_OK && !self && n > 0) rc = ar.alloc(&dr, (size_t)n * d);
    if (rc == KNN_OK) rc = ar.alloc(&di, (size_t)m * k);
    if (rc == KNN_OK) rc = ar.alloc(&dd, (size_t)m * k);
    if (self) dr = dq;
    cudaError_t e = cudaSuccess;
    if (rc == KNN_OK)
      e = cudaMemcpyAsync(dq, q, sizeof(float) * m * d, cudaMemcpyHostToDevice, s);
    if (rc == KNN_OK && e == cudaSuccess && !self && n > 0)
      e = cudaMemcpyAsync(dr, r, sizeof(float) * n * d, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      set_error("host-to-device copy failed: %s", cudaGetErrorString(e));
      rc = KNN_ECUDA;
    }
    if (rc == KNN_OK) {
      // always the synchronising path, which also checks the device error flag
      knn_stats local;
      rc = join_device_impl(dq, m, dr, n, d, k, di, dd, opt, st ? st : &local, s, &sink);
    }
    if (rc == KNN_OK && !sink.done) {
      e = cudaMemcpyAsync(out_idx, di, sizeof(int32_t) * m * k,
                          cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_dist, dd, sizeof(float) * m * k,
                            cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) {
        set_error("device-to-host copy failed: %s", cudaGetErrorString(e));
        rc = KNN_ECUDA;
      }
    }
    // the result buffers are released on `s` when the arena closes: the
    // chunk copies on `cs` must have finished by then
    cudaError_t ec = cudaStreamSynchronize(cs);
    if (ec != cudaSuccess && rc == KNN_OK) {
      set_error("device-to-host copy failed: %s", cudaGetErrorString(ec));
      rc = KNN_ECUDA;
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess && rc == KNN_OK) {
    set_error("join failed on the device: %s", cudaGetErrorString(e));
    rc = KNN_ECUDA;
  }
  return rc;
}

int knn_trim_memory(void) {
  error_buffer().clear();
  std::lock_guard<std::mutex> guard(g_pool_mu);
  for (int d = 0; d < kMaxDevices; d++) {
    if (!g_pools[d]) continue;
    cudaError_t e = cudaMemPoolTrimTo(g_pools[d], 0);
    if (e != cudaSuccess) {
      set_error("cudaMemPoolTrimTo failed: %s", cudaGetErrorString(e));
      return KNN_ECUDA;
    }
  }
  return KNN_OK;
}

void knn_pack_indexdist(const int32_t *idx, const float *dist, int64_t count,
                        void *out) {
  if (!idx || !dist || !out) return;
  uint32_t *o = static_cast<uint32_t *>(out);
  for (int64_t i = 0; i < count; i++) {
    uint32_t b;
    memcpy(&b, dist + i, 4);
    o[2 * i] = (uint32_t)idx[i];
    o[2 * i + 1] = b;
  }
}

}  // extern "C"

// Test hook (not part of the public ABI): the representative rows the
// seeded draw picks (the reference's 10-trial spread selection,
// src/knnjoin.cu:195-239, 125-154) for device points pts (n x d floats);
// rows_out is a device array of R ints.
extern "C" int knnsweet_test_select_reps(const float *pts, int64_t n, int32_t d, int32_t R,
                                         uint32_t seed, int32_t trials, int32_t *rows_out) {
  using namespace knnsweet;
  error_buffer().clear();
  if (!pts || !rows_out || n <= 0 || d <= 0 || R <= 0 || R > n || trials <= 0) {
    set_error("bad arguments");
    return KNN_EINVAL;
  }
  cudaStream_t s = 0;
  int rc = KNN_OK;
  {
    Arena ar(s);
    const int dp4 = (d + 3) / 4;
    float4 *rows = nullptr, *reps = nullptr;
    int32_t *cand = nullptr;
    uint32_t *score = nullptr;
    std::vector<int32_t> draw((size_t)trials * R);
    GlibcRand g(seed);
    for (auto &c : draw) c = g.next() % (int32_t)n;
    rc = ar.alloc(&rows, (size_t)n * dp4);
    if (rc == KNN_OK) rc = ar.alloc(&reps, (size_t)R * dp4);
    if (rc == KNN_OK) rc = ar.alloc(&cand, draw.size());
    if (rc == KNN_OK) rc = ar.alloc(&score, (size_t)trials);
    if (rc == KNN_OK) rc = launch_pack_rows(pts, n, d, dp4, rows, s);
    if (rc == KNN_OK) rc = upload_i32(draw, cand, s);
    if (rc == KNN_OK) rc = launch_rep_select(rows, dp4, cand, R, trials, score, reps, rows_out, s);
  }
  if (rc == KNN_OK && cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("device failure");
    rc = KNN_ECUDA;
  }
  return rc;
}
