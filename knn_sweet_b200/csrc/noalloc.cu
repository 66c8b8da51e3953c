// noalloc.cu -- the exact kNN join for callers that may not allocate device
// memory (knn_join_device_noalloc in include/knnsweet.h).
//
// Who needs it: applications that reserve the whole GPU for their own memory
// manager at start-up (a serving or database process that hands out device
// memory only through its own allocator) and code that is not allowed to
// allocate once it is running, because cudaMalloc / cudaFree can block and
// synchronise the device at an unpredictable moment.  Such a caller still
// owns its inputs and outputs; everything else the join needs lives in one
// fixed array compiled into this library.
//
// The join is knn_join_device's plain FP32 pipeline with the reference's
// representative draw (same kernels, same launch order, same results); only
// the origin of the scratch differs: every buffer is carved from
// `g_static_scratch` instead of the stream-ordered pool, and the draw reaches
// the device as kernel parameters, so no host heap is touched either.  The
// BF16 form and the representative refinement are refused (their buffers
// scale with options this array cannot promise).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "glibc_rand.h"
#include "kernels.cuh"

// Scratch shared by every knn_join_device_noalloc call on a device.  Each
// GPU that loads this library's code holds it until the process exits.
static __device__ __align__(256) unsigned char g_static_scratch[KNN_NOALLOC_SCRATCH_BYTES];

namespace knnsweet {

int check_sizes(int64_t m, int64_t n, int32_t d, int32_t k);
int check_options(const knn_options *opt, knn_options *o);

namespace {

// Device address of g_static_scratch per device.  In host code the symbol
// names a host-side stand-in, not device memory, so it is never handed to a
// kernel directly: the address comes from cudaGetSymbolAddress, taken once
// per device with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
unsigned char *g_addr[kMaxDevices] = {};

int static_scratch(unsigned char **out) {
  int dev = 0;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d out of range", dev);
    return KNN_EINVAL;
  }
  std::lock_guard<std::mutex> guard(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaGetSymbolAddress(static scratch) failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return KNN_ECUDA;
    }
    g_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_addr[dev];
  return KNN_OK;
}

// Bump allocation over the fixed array; with a null base it only measures.
class Carver {
 public:
  explicit Carver(unsigned char *base) : base_(base) {}
  template <class T>
  T *take(int64_t count) {
    const size_t off = (used_ + 255) & ~(size_t)255;
    used_ = off + (size_t)(count > 0 ? count : 1) * sizeof(T);
    return base_ ? reinterpret_cast<T *>(base_ + off) : nullptr;
  }
  size_t used() const { return used_; }

 private:
  unsigned char *base_;
  size_t used_ = 0;
};

struct SideBufs {
  float4 *packed = nullptr;  // null: the input rows are used in place
  int32_t *cand = nullptr;
  uint32_t *score = nullptr;
  float4 *reps = nullptr;
  int32_t *rep_rows = nullptr;
  int32_t *cl = nullptr;
  float *dr = nullptr;
  uint64_t *keys = nullptr, *skeys = nullptr;
  int32_t *vals = nullptr, *perm = nullptr;
  unsigned char *temp = nullptr;
  size_t temp_bytes = 0;
  unsigned char *tc = nullptr;  // tensor-core assignment scratch (d >= 16)
  int32_t *off = nullptr;
};

// Device counters: [0] scan work counter, [1 ..] scan statistics, then the
// count of queries left to the band kernel, the device error flag and the
// two sides' exactness flags.
constexpr int kCtrUnres = 1 + kScanCounters, kCtrErr = kCtrUnres + 1;
constexpr int kCtrInexactR = kCtrErr + 1, kCtrInexactQ = kCtrErr + 2, kCtrCount = kCtrErr + 3;

struct Plan {
  int64_t m = 0, n = 0;
  int d = 0, k = 0, dp4s = 0, tmpl = 0, Rq = 0, Rs = 0, trials = 0;
  uint32_t seed = 0;
  bool share = false, pack_r = false, pack_q = false, idx_in_row = false, use_tc = false;
  SideBufs S, Q;
  float4 *srows = nullptr;
  float *sdist = nullptr, *cmin = nullptr, *cmax = nullptr;
  int32_t *sidx = nullptr;
  float *qrad = nullptr, *drr = nullptr, *theta0 = nullptr;
  int32_t *slot_cl = nullptr, *rlist = nullptr, *rlen = nullptr;
  int32_t *unres = nullptr;
  unsigned long long *ctr = nullptr;
};

void carve_side(Carver &c, SideBufs &b, int64_t n, int d, int dp4s, int R, int trials, bool pack,
                bool use_tc) {
  b.packed = pack ? c.take<float4>(n * dp4s) : nullptr;
  b.cand = c.take<int32_t>((int64_t)trials * R);
  b.score = c.take<uint32_t>(trials);
  b.reps = c.take<float4>((int64_t)R * dp4s);
  b.rep_rows = c.take<int32_t>(R);
  b.cl = c.take<int32_t>(n);
  b.dr = c.take<float>(n);
  b.keys = c.take<uint64_t>(n);
  b.vals = c.take<int32_t>(n);
  b.skeys = c.take<uint64_t>(n);
  b.perm = c.take<int32_t>(n);
  b.temp_bytes = cluster_sort_temp_bytes(n, R);
  b.temp = c.take<unsigned char>((int64_t)b.temp_bytes);
  b.tc = use_tc ? c.take<unsigned char>((int64_t)assign_tc_scratch_bytes(R, d)) : nullptr;
  b.off = c.take<int32_t>((int64_t)R + 1);
}

void carve(Carver &c, Plan &p) {
  carve_side(c, p.S, p.n, p.d, p.dp4s, p.Rs, p.trials, p.pack_r, p.use_tc);
  p.srows = c.take<float4>(p.n * p.dp4s);
  p.sdist = c.take<float>(p.n);
  p.sidx = c.take<int32_t>(p.n);
  p.cmin = c.take<float>(p.Rs);
  p.cmax = c.take<float>(p.Rs);
  if (!p.share) carve_side(c, p.Q, p.m, p.d, p.dp4s, p.Rq, p.trials, p.pack_q, p.use_tc);
  p.qrad = c.take<float>(p.Rq);
  p.slot_cl = c.take<int32_t>(p.m);
  p.drr = c.take<float>((int64_t)p.Rq * p.Rs);
  p.theta0 = c.take<float>(p.Rq);
  p.rlist = c.take<int32_t>((int64_t)p.Rq * p.Rs);
  p.rlen = c.take<int32_t>(p.Rq);
  p.unres = c.take<int32_t>(p.m);
  p.ctr = c.take<unsigned long long>(kCtrCount);
}

// The representative draw travels as kernel parameters, 8,000 indices per
// launch, from a chunk on the host stack.
struct DrawChunk {
  int32_t count;
  int32_t v[8000];
};

__global__ void draw_upload_kernel(int32_t *__restrict__ dst, const DrawChunk c) {
  for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[i] = c.v[i];
}

__global__ void noalloc_fill_empty_kernel(int32_t *idx, float *dist, int64_t count) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    idx[t] = -1;
    dist[t] = __int_as_float(0x7f800000);
  }
}

int draw_reps(const SideBufs &b, int64_t n, int R, int trials, uint32_t seed,
              cudaStream_t s) {
  DrawChunk chunk;
  GlibcRand g(seed);
  const int64_t total = (int64_t)trials * R;
  for (int64_t done = 0; done < total;) {
    const int cnt = (int)(total - done < 8000 ? total - done : 8000);
    for (int i = 0; i < cnt; i++) chunk.v[i] = g.next() % (int32_t)n;
    chunk.count = cnt;
    draw_upload_kernel<<<1, 256, 0, s>>>(b.cand + done, chunk);
    KNN_LAUNCH_CHECK();
    done += cnt;
  }
  return KNN_OK;
}

int cluster_side(const Plan &p, const SideBufs &b, const float *src, int64_t n, int R,
                 const float4 **rows_out, cudaStream_t s) {
  const float4 *rows = reinterpret_cast<const float4 *>(src);
  if (b.packed) {
    int rc = launch_pack_rows(src, n, p.d, p.dp4s, b.packed, s);
    if (rc != KNN_OK) return rc;
    rows = b.packed;
  }
  int rc = draw_reps(b, n, R, p.trials, p.seed, s);
  if (rc == KNN_OK)
    rc = launch_rep_select(rows, p.dp4s, b.cand, R, p.trials, b.score, b.reps, b.rep_rows, s);
  if (rc == KNN_OK) {
    if (b.tc)
      rc = launch_assign_tc(rows, n, p.dp4s, p.d, b.reps, R, b.tc, b.cl, b.dr,
                            reinterpret_cast<int *>(p.ctr + kCtrErr), s);
    else
      rc = launch_assign(rows, n, p.dp4s, b.reps, R, b.cl, b.dr, s);
  }
  if (rc == KNN_OK)
    rc = launch_cluster_sort(b.cl, b.dr, n, R, b.keys, b.vals, b.skeys, b.perm, b.temp,
                             b.temp_bytes, s);
  if (rc == KNN_OK) rc = launch_cluster_offsets(b.skeys, n, R, b.off, s);
  *rows_out = rows;
  return rc;
}

int reps_for(int64_t n) {  // same default as knn_join_device
  double r = std::floor(1.6 * std::sqrt((double)n) + 0.5);
  return (int)(r < 1 ? 1 : (r > 4096 ? 4096 : r));
}

int noalloc_join(const float *q, int64_t m, const float *r, int64_t n, int32_t d, int32_t k,
                 int32_t *out_idx, float *out_dist, const knn_options *opt,
                 cudaStream_t s) {
  knn_options o;
  int rc = check_options(opt, &o);
  if (rc == KNN_OK) rc = check_sizes(m, n, d, k);
  if (rc != KNN_OK) return rc;
  if (o.precision != KNN_FP32) {
    set_error("knn_join_device_noalloc: precision must be KNN_FP32 (the BF16 form's "
              "candidate buffers grow with k and margin beyond the fixed scratch)");
    return KNN_EINVAL;
  }
  if (o.lloyd_iters != 0) {
    set_error("knn_join_device_noalloc: lloyd_iters must be 0 (representative refinement "
              "is only available through knn_join_device)");
    return KNN_EINVAL;
  }
  launch_counter() = 0;
  if (m == 0) return KNN_OK;
  if (!q || (!r && n > 0) || !out_idx || !out_dist) {
    set_error("null pointer argument");
    return KNN_EINVAL;
  }
  if (n == 0) {
    noalloc_fill_empty_kernel<<<256, 256, 0, s>>>(out_idx, out_dist, m * (int64_t)k);
    KNN_LAUNCH_CHECK();
    return KNN_OK;
  }

  Plan p;
  p.m = m;
  p.n = n;
  p.d = d;
  p.k = k;
  const int dp4 = (d + 3) / 4;
  p.dp4s = dp4;
  if (dp4 <= 8) {
    p.dp4s = 1;
    while (p.dp4s < dp4) p.dp4s <<= 1;
    p.tmpl = p.dp4s;
  }
  const bool self = (q == r) && (m == n);
  p.Rs = o.sreps > 0 ? o.sreps : reps_for(n);
  p.Rq = o.qreps > 0 ? o.qreps : (self ? p.Rs : reps_for(m));
  if (p.Rs > n) p.Rs = (int)n;
  if (p.Rq > m) p.Rq = (int)m;
  p.share = self && p.Rq == p.Rs;
  p.trials = o.rep_trials;
  p.seed = o.seed;
  p.idx_in_row = p.tmpl > 0 && 4 * p.dp4s > d;
  auto needs_pack = [&](const float *src) {
    return !(p.dp4s * 4 == d && (reinterpret_cast<uintptr_t>(src) & 15) == 0);
  };
  p.pack_r = needs_pack(r);
  p.pack_q = needs_pack(q);
  p.use_tc = (o.flags & KNN_NO_TENSOR_CORES) == 0 && assign_tc_supported(d);

  // size check before anything touches the array
  Carver measure(nullptr);
  carve(measure, p);
  if (measure.used() > (size_t)KNN_NOALLOC_SCRATCH_BYTES) {
    set_error("join of m=%lld, n=%lld, d=%d, k=%d with %d/%d representatives needs %zu "
              "bytes of scratch; the allocation-free entry point has %zu",
              (long long)m, (long long)n, d, k, p.Rq, p.Rs, measure.used(),
              (size_t)KNN_NOALLOC_SCRATCH_BYTES);
    return KNN_EINVAL;
  }
  unsigned char *base = nullptr;
  rc = static_scratch(&base);
  if (rc != KNN_OK) return rc;
  Carver carver(base);
  carve(carver, p);

  int dev = 0, num_sms = 148;
  KNN_CUDA_TRY(cudaGetDevice(&dev));
  KNN_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));

  // the array keeps the previous call's contents: the counters (work
  // counter, statistics, band list length, error flag) must start at zero;
  // every other buffer is written before it is read
  KNN_CUDA_TRY(cudaMemsetAsync(p.ctr, 0, kCtrCount * sizeof(unsigned long long), s));
  const float4 *Rp = nullptr, *Qp = nullptr;
  rc = cluster_side(p, p.S, r, n, p.Rs, &Rp, s);
  if (rc != KNN_OK) return rc;
  rc = launch_cluster_layout(p.S.skeys, p.S.perm, n, Rp, p.dp4s, p.idx_in_row, p.srows,
                             p.sdist, p.sidx, s);
  if (rc == KNN_OK) rc = launch_cluster_minmax(p.S.off, p.sdist, p.Rs, p.cmin, p.cmax, s);
  if (rc != KNN_OK) return rc;
  const SideBufs &Qb = p.share ? p.S : p.Q;
  if (p.share) {
    Qp = Rp;
  } else {
    rc = cluster_side(p, p.Q, q, m, p.Rq, &Qp, s);
    if (rc != KNN_OK) return rc;
  }
  rc = launch_query_clusters(Qb.skeys, Qb.off, m, p.Rq, p.qrad, p.slot_cl, s);
  if (rc == KNN_OK) rc = launch_rep_dist(Qb.reps, p.Rq, p.S.reps, p.Rs, p.dp4s, p.drr, s);
  if (rc == KNN_OK)
    rc = launch_bounds_filter(p.drr, p.Rq, p.Rs, p.qrad, Qb.off, p.S.off, p.sdist, p.cmax,
                              k, d, p.theta0, p.rlist, p.rlen, nullptr, s);
  if (rc != KNN_OK) return rc;
  ScanArgs a{};
  a.qrows = Qp;
  a.qorder = Qb.perm;
  a.slot_cl = p.slot_cl;
  a.m = m;
  a.d = d;
  a.dp4 = p.dp4s;
  a.dp4_tmpl = p.tmpl;
  a.k = k;
  a.idx_in_row = p.idx_in_row;
  a.squared = (o.flags & KNN_SQUARED_DIST) != 0;
  a.sreps = p.S.reps;
  a.srows = p.srows;
  a.sdist = p.sdist;
  a.sidx = p.sidx;
  a.soff = p.S.off;
  a.cmin = p.cmin;
  a.cmax = p.cmax;
  a.theta0 = p.theta0;
  a.qrad = p.qrad;
  a.qkeys = Qb.skeys;
  a.rlist = p.rlist;
  a.rlen = p.rlen;
  a.Rs = p.Rs;
  a.n_ref = n;
  a.rrows = Rp;
  {
    int *fr = reinterpret_cast<int *>(p.ctr + kCtrInexactR);
    int *fq = reinterpret_cast<int *>(p.ctr + kCtrInexactQ);
    rc = launch_exact_check(reinterpret_cast<const float *>(Rp), n * p.dp4s * 4, d, fr, s);
    if (rc == KNN_OK && !p.share)
      rc = launch_exact_check(reinterpret_cast<const float *>(Qp), m * p.dp4s * 4, d, fq, s);
    if (rc != KNN_OK) return rc;
    a.inexact_r = fr;
    a.inexact_q = p.share ? fr : fq;
  }
  a.out_idx = out_idx;
  a.out_dist = out_dist;
  a.unres_slot = p.unres;
  a.unres_count = reinterpret_cast<unsigned *>(p.ctr + kCtrUnres);
  a.work_counter = p.ctr;
  a.counters = p.ctr + 1;
  return launch_scan(a, num_sms, s);
}

}  // namespace
}  // namespace knnsweet

extern "C" int knn_join_device_noalloc(const float *q, int64_t m, const float *r,
                                       int64_t n, int32_t d, int32_t k, int32_t *out_idx,
                                       float *out_dist, const knn_options *opt,
                                       void *stream) {
  knnsweet::error_buffer().clear();
  return knnsweet::noalloc_join(q, m, r, n, d, k, out_idx, out_dist, opt,
                                static_cast<cudaStream_t>(stream));
}
