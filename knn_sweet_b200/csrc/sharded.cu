// sharded.cu -- the join over several GPUs: one process driving a list of
// devices (knn_join_sharded), or one process per GPU each taking its part
// (knn_join_partition_device).
//
// The reference runs its whole search on one GPU (src/knnjoin.cu:1103-1129).
// Queries are independent, so the search shards with no exchange during it;
// what is split is the set of QUERY CLUSTERS, in contiguous ranges of the
// cluster order balanced by an estimate of their work (query count times the
// band sizes they can scan, launch_cluster_work), so a query cluster -- whose
// queries walk the same candidate list -- never straddles two devices and a
// skewed cluster size distribution does not leave devices idle.
//
// knn_join_sharded builds the reference index and the query side ONCE, on
// the first listed device, then copies what the search reads (rows, member
// lists, bounds, candidate lists: N (4 dp4 + 12) bytes and Rq Rs 4 bytes of
// lists) to every other device with peer copies over NVLink.  Each device
// searches its range and stores its results directly into the first
// device's result buffer through peer memory (plain stores from the scan
// kernels, no multicast); where peer access is not available a device
// searches into a local buffer that is copied back and merged by rows.
#include <algorithm>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "pipeline.cuh"

namespace knnsweet {
namespace {

// Contiguous ranges of query clusters, cut where the prefix sum of the
// estimated work crosses g / parts of the total: cut[g] .. cut[g+1]-1 is
// part g (cut[0] = 0, cut[parts] = Rq).
std::vector<int> partition_clusters(const std::vector<long long> &work, int parts) {
  const int Rq = (int)work.size();
  std::vector<long long> pre(Rq + 1, 0);
  for (int c = 0; c < Rq; c++) pre[c + 1] = pre[c] + work[c];
  std::vector<int> cut(parts + 1, Rq);
  cut[0] = 0;
  for (int g = 1; g < parts; g++) {
    const long double target = (long double)pre[Rq] * g / parts;
    int c = (int)(std::lower_bound(pre.begin(), pre.end(), (long long)target) - pre.begin());
    cut[g] = std::max(cut[g - 1], std::min(c, Rq));
  }
  return cut;
}

// Work estimate and partition of a built join (synchronises `s`); qoff_h
// gets the query clusters' slot offsets.
int plan_parts(const RefSide &R, const QuerySide &Q, int parts, Arena &ar, cudaStream_t s,
               std::vector<int> *cut, std::vector<int32_t> *qoff_h) {
  const int Rq = Q.Rq;
  long long *work;
  KNN_TRY(ar.alloc(&work, (size_t)Rq));
  KNN_TRY(launch_cluster_work(Q.drr, Rq, R.Rs, Q.qrad, Q.theta0, Q.qset.off, Q.rlist, Q.rlen,
                              R.sset.off, R.sdist, work, s));
  std::vector<long long> w(Rq);
  qoff_h->assign(Rq + 1, 0);
  KNN_CUDA_TRY(cudaMemcpyAsync(w.data(), work, sizeof(long long) * Rq, cudaMemcpyDeviceToHost, s));
  KNN_CUDA_TRY(cudaMemcpyAsync(qoff_h->data(), Q.qset.off, sizeof(int32_t) * (Rq + 1),
                               cudaMemcpyDeviceToHost, s));
  KNN_CUDA_TRY(cudaStreamSynchronize(s));
  *cut = partition_clusters(w, parts);
  return KNN_OK;
}

// Rows of the slots slot0 .. slot0+nslot-1 (queries qorder[slot]) from src
// to dst (both m x k).
__global__ void merge_rows_kernel(const int32_t *__restrict__ qorder, int64_t slot0,
                                  int64_t nslot, int k, const int32_t *__restrict__ si,
                                  const float *__restrict__ sd, int32_t *__restrict__ di,
                                  float *__restrict__ dd) {
  const int64_t total = nslot * k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = qorder[slot0 + t / k];
    const int64_t e = q * k + t % k;
    di[e] = si[e];
    dd[e] = sd[e];
  }
}

// A copy of `count` elements of a device-0 array on device g.
template <class T>
int replicate(Arena &ar, int g, int g0, const T *src, size_t count, cudaStream_t s, T **out) {
  *out = nullptr;
  if (!src) return KNN_OK;
  T *p;
  KNN_TRY(ar.alloc(&p, count));
  KNN_CUDA_TRY(cudaMemcpyPeerAsync(p, g, src, g0, count * sizeof(T), s));
  *out = p;
  return KNN_OK;
}

// What the search reads of R and Q, copied to device g.
int replicate_sides(Arena &ar, int g, int g0, const RefSide &R, const QuerySide &Q, int64_t m,
                    bool share, cudaStream_t s, RefSide *R2, QuerySide *Q2) {
  const int64_t n = R.n;
  const int dp4 = R.dp4s, Rs = R.Rs, Rq = Q.Rq;
  *R2 = RefSide{};
  R2->n = n;
  R2->d = R.d;
  R2->dp4s = dp4;
  R2->tmpl = R.tmpl;
  R2->Rs = Rs;
  R2->idx_in_row = R.idx_in_row;
  R2->sset.R = Rs;
  float4 *rp;
  KNN_TRY(replicate(ar, g, g0, R.Rp, (size_t)n * dp4, s, &rp));
  R2->Rp = rp;
  KNN_TRY(replicate(ar, g, g0, R.sset.reps, (size_t)Rs * dp4, s, &R2->sset.reps));
  KNN_TRY(replicate(ar, g, g0, R.sset.off, (size_t)Rs + 1, s, &R2->sset.off));
  KNN_TRY(replicate(ar, g, g0, R.srows, (size_t)n * dp4, s, &R2->srows));
  KNN_TRY(replicate(ar, g, g0, R.sdist, (size_t)n, s, &R2->sdist));
  KNN_TRY(replicate(ar, g, g0, R.sidx, (size_t)n, s, &R2->sidx));
  KNN_TRY(replicate(ar, g, g0, R.cmin, (size_t)Rs, s, &R2->cmin));
  KNN_TRY(replicate(ar, g, g0, R.cmax, (size_t)Rs, s, &R2->cmax));
  KNN_TRY(replicate(ar, g, g0, R.inexact, 1, s, &R2->inexact));
  *Q2 = QuerySide{};
  Q2->Rq = Rq;
  if (share) {
    Q2->Qp = R2->Rp;
    Q2->inexact = R2->inexact;
  } else {
    float4 *qp;
    int *qf;
    KNN_TRY(replicate(ar, g, g0, Q.Qp, (size_t)m * dp4, s, &qp));
    KNN_TRY(replicate(ar, g, g0, Q.inexact, 1, s, &qf));
    Q2->Qp = qp;
    Q2->inexact = qf;
  }
  Q2->qset.R = Rq;
  KNN_TRY(replicate(ar, g, g0, Q.qset.perm, (size_t)m, s, &Q2->qset.perm));
  KNN_TRY(replicate(ar, g, g0, Q.qset.off, (size_t)Rq + 1, s, &Q2->qset.off));
  KNN_TRY(replicate(ar, g, g0, Q.slot_cl, (size_t)m, s, &Q2->slot_cl));
  KNN_TRY(replicate(ar, g, g0, Q.theta0, (size_t)Rq, s, &Q2->theta0));
  KNN_TRY(replicate(ar, g, g0, Q.qrad, (size_t)Rq, s, &Q2->qrad));
  KNN_TRY(replicate(ar, g, g0, Q.qset.skeys, (size_t)m, s, &Q2->qset.skeys));
  KNN_TRY(replicate(ar, g, g0, Q.rlist, (size_t)Rq * Rs, s, &Q2->rlist));
  KNN_TRY(replicate(ar, g, g0, Q.rlen, (size_t)Rq, s, &Q2->rlen));
  if (Q.clb)
    KNN_TRY(replicate(ar, g, g0, Q.clb, (size_t)Rq * ((Rs + 31) / 32), s, &Q2->clb));
  return KNN_OK;
}

// One shard of knn_join_sharded: its device, stream, arena and range.
struct Shard {
  int device = 0;
  int c0 = 0, c1 = 0;
  int64_t slot0 = 0, nslot = 0;
  cudaStream_t s = nullptr;
  Arena *ar = nullptr;
  unsigned long long *ctr = nullptr;
  int32_t *li = nullptr;  // local result buffers (no peer access)
  float *ld = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

int sharded_impl(const float *q, int64_t m, const float *r, int64_t n, int32_t d, int32_t k,
                 int32_t *out_idx, float *out_dist, const knn_options &o,
                 const int32_t *devices, int32_t ndev, knn_stats *st) {
  const int g0 = devices[0];
  KNN_CUDA_TRY(cudaSetDevice(g0));
  cudaStream_t s0;
  KNN_CUDA_TRY(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
  std::vector<Shard> sh(ndev);
  int rc = KNN_OK;
  {
    Arena ar0(s0);
    auto body = [&]() -> int {
      const bool self = q == r && m == n;
      int Rs = o.sreps > 0 ? o.sreps : default_reps(n);
      if (Rs > n) Rs = (int)n;
      const int Rq = query_rep_count(o, m, d, k, self, Rs);
      const bool share = self && Rq == Rs;
      cudaEvent_t e_build[2] = {nullptr, nullptr};
      struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard() {
          for (int i = 0; i < 2; i++)
            if (e[i]) cudaEventDestroy(e[i]);
        }
      } guard{e_build};
      KNN_CUDA_TRY(cudaEventCreate(&e_build[0]));
      KNN_CUDA_TRY(cudaEventCreate(&e_build[1]));
      KNN_CUDA_TRY(cudaEventRecord(e_build[0], s0));
      // inputs on the first device; the index and the query side built there
      float *dq, *dr, *od0f;
      int32_t *oi0i;
      unsigned long long *ctr0;
      KNN_TRY(ar0.alloc(&ctr0, kCtrCount));
      KNN_CUDA_TRY(cudaMemsetAsync(ctr0, 0, kCtrCount * sizeof(unsigned long long), s0));
      KNN_TRY(ar0.alloc(&dq, (size_t)m * d));
      KNN_CUDA_TRY(cudaMemcpyAsync(dq, q, sizeof(float) * m * d, cudaMemcpyHostToDevice, s0));
      if (self) {
        dr = dq;
      } else {
        KNN_TRY(ar0.alloc(&dr, (size_t)n * d));
        KNN_CUDA_TRY(cudaMemcpyAsync(dr, r, sizeof(float) * n * d, cudaMemcpyHostToDevice, s0));
      }
      KNN_TRY(ar0.alloc(&oi0i, (size_t)m * k));
      KNN_TRY(ar0.alloc(&od0f, (size_t)m * k));
      RefSide R;
      KNN_TRY(build_ref_side(ar0, ar0, dr, n, d, Rs, o, false,
                             reinterpret_cast<int *>(ctr0 + kCtrErr), s0, &R));
      QuerySide Q;
      KNN_TRY(build_query_side(R, share, dq, m, k, o, ar0, ctr0, s0, &Q));
      std::vector<int> cut;
      std::vector<int32_t> qoff;
      KNN_TRY(plan_parts(R, Q, ndev, ar0, s0, &cut, &qoff));
      KNN_CUDA_TRY(cudaEventRecord(e_build[1], s0));
      // one replica of the search's inputs per further device
      std::vector<int> rep_dev;
      std::vector<RefSide> rep_R;
      std::vector<QuerySide> rep_Q;
      std::vector<cudaEvent_t> rep_ev;  // a replica is complete
      struct RepEvGuard {
        std::vector<cudaEvent_t> *v;
        ~RepEvGuard() {
          for (cudaEvent_t e : *v) cudaEventDestroy(e);
        }
      } rep_guard{&rep_ev};
      for (int i = 0; i < ndev; i++) {
        Shard &x = sh[i];
        x.device = devices[i];
        x.c0 = cut[i];
        x.c1 = cut[i + 1];
        x.slot0 = qoff[x.c0];
        x.nslot = qoff[x.c1] - qoff[x.c0];
        KNN_CUDA_TRY(cudaSetDevice(x.device));
        KNN_CUDA_TRY(cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking));
        x.ar = new Arena(x.s);
        KNN_CUDA_TRY(cudaEventCreate(&x.ev[0]));
        KNN_CUDA_TRY(cudaEventCreate(&x.ev[1]));
        KNN_CUDA_TRY(cudaStreamWaitEvent(x.s, e_build[1], 0));
        KNN_CUDA_TRY(cudaEventRecord(x.ev[0], x.s));
        KNN_TRY(x.ar->alloc(&x.ctr, kCtrCount));
        KNN_CUDA_TRY(cudaMemsetAsync(x.ctr, 0, kCtrCount * sizeof(unsigned long long), x.s));
      }
      for (int i = 0; i < ndev; i++) {
        Shard &x = sh[i];
        if (x.nslot == 0) continue;
        KNN_CUDA_TRY(cudaSetDevice(x.device));
        const RefSide *Rx = &R;
        const QuerySide *Qx = &Q;
        int32_t *oi = oi0i;
        float *od = od0f;
        if (x.device != g0) {
          int j = (int)(std::find(rep_dev.begin(), rep_dev.end(), x.device) - rep_dev.begin());
          if (j == (int)rep_dev.size()) {
            rep_dev.push_back(x.device);
            rep_R.emplace_back();
            rep_Q.emplace_back();
            KNN_TRY(replicate_sides(*x.ar, x.device, g0, R, Q, m, share, x.s, &rep_R.back(),
                                    &rep_Q.back()));
            cudaEvent_t ev;
            KNN_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            rep_ev.push_back(ev);
            KNN_CUDA_TRY(cudaEventRecord(ev, x.s));
          } else {
            // shards of one device run on their own streams: a later shard
            // waits for the replica the first one copied
            KNN_CUDA_TRY(cudaStreamWaitEvent(x.s, rep_ev[j], 0));
          }
          Rx = &rep_R[j];
          Qx = &rep_Q[j];
          int can = 0;
          KNN_CUDA_TRY(cudaDeviceCanAccessPeer(&can, x.device, g0));
          if (can) {
            cudaError_t e = cudaDeviceEnablePeerAccess(g0, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            else if (e != cudaSuccess) can = 0, cudaGetLastError();
          }
          if (!can) {
            KNN_TRY(x.ar->alloc(&x.li, (size_t)m * k));
            KNN_TRY(x.ar->alloc(&x.ld, (size_t)m * k));
            oi = x.li;
            od = x.ld;
          }
        }
        KNN_TRY(search_clusters(*Rx, *Qx, m, k, x.c0, x.c1, x.slot0, x.nslot, oi, od, o, x.s,
                                nullptr, *x.ar, x.ctr));
        KNN_CUDA_TRY(cudaEventRecord(x.ev[1], x.s));
      }
      // a later shard on a replicated device used the first shard's replica:
      // the replicas are complete once every stream is done
      for (int i = 0; i < ndev; i++) {
        KNN_CUDA_TRY(cudaSetDevice(sh[i].device));
        KNN_CUDA_TRY(cudaStreamSynchronize(sh[i].s));
      }
      // shards without peer access: their rows merged on the first device
      KNN_CUDA_TRY(cudaSetDevice(g0));
      for (const Shard &x : sh) {
        if (!x.li) continue;
        int32_t *ti;
        float *td;
        KNN_TRY(ar0.alloc(&ti, (size_t)m * k));
        KNN_TRY(ar0.alloc(&td, (size_t)m * k));
        KNN_CUDA_TRY(cudaMemcpyPeerAsync(ti, g0, x.li, x.device, sizeof(int32_t) * m * k, s0));
        KNN_CUDA_TRY(cudaMemcpyPeerAsync(td, g0, x.ld, x.device, sizeof(float) * m * k, s0));
        merge_rows_kernel<<<1024, 256, 0, s0>>>(Q.qset.perm, x.slot0, x.nslot, k, ti, td, oi0i,
                                                od0f);
        KNN_LAUNCH_CHECK();
      }
      KNN_CUDA_TRY(cudaMemcpyAsync(out_idx, oi0i, sizeof(int32_t) * m * k,
                                   cudaMemcpyDeviceToHost, s0));
      KNN_CUDA_TRY(cudaMemcpyAsync(out_dist, od0f, sizeof(float) * m * k,
                                   cudaMemcpyDeviceToHost, s0));
      KNN_CUDA_TRY(cudaStreamSynchronize(s0));
      if (st) {
        memset(st, 0, sizeof *st);
        KNN_TRY(read_stats(ctr0, s0, st));  // the build's device error flag
        KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_build, e_build[0], e_build[1]));
        for (const Shard &x : sh) {
          KNN_CUDA_TRY(cudaSetDevice(x.device));
          KNN_TRY(read_stats(x.ctr, x.s, st));
          float ms = 0.0f;
          if (x.nslot > 0) KNN_CUDA_TRY(cudaEventElapsedTime(&ms, x.ev[0], x.ev[1]));
          st->ms_search = std::max(st->ms_search, ms);
        }
        st->ms_total = st->ms_build + st->ms_search;
        st->pairs_total = m * n;
        st->pairs_pruned = st->pairs_total - st->dist_evals;
        st->qreps_used = Q.Rq;
        st->sreps_used = R.Rs;
        st->kernels_launched = launch_counter();
      }
      return KNN_OK;
    };
    rc = body();
    // release every shard's scratch on its own device before the first
    // device's, once no stream runs (a shard may read another shard's
    // replica and the first device's buffers)
    for (Shard &x : sh) {
      if (!x.s) continue;
      cudaSetDevice(x.device);
      cudaStreamSynchronize(x.s);
    }
    for (Shard &x : sh) {
      if (!x.s) continue;
      cudaSetDevice(x.device);
      delete x.ar;
      x.ar = nullptr;
      cudaStreamSynchronize(x.s);
      for (cudaEvent_t e : x.ev)
        if (e) cudaEventDestroy(e);
      cudaStreamDestroy(x.s);
    }
    cudaSetDevice(g0);
  }
  cudaStreamSynchronize(s0);
  cudaStreamDestroy(s0);
  return rc;
}

}  // namespace
}  // namespace knnsweet

using namespace knnsweet;

extern "C" int knn_join_sharded(const float *q, int64_t m, const float *r, int64_t n,
                                int32_t d, int32_t k, int32_t *out_idx, float *out_dist,
                                const knn_options *opt, const int32_t *devices, int32_t ndev,
                                knn_stats *st) {
  error_buffer().clear();
  launch_counter() = 0;
  if (st) memset(st, 0, sizeof *st);
  knn_options o;
  int rc = check_options(opt, &o);
  if (rc == KNN_OK) rc = check_sizes(m, n, d, k);
  if (rc != KNN_OK) return rc;
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
  int prev = 0;
  cudaGetDevice(&prev);
  rc = sharded_impl(q, m, r, n, d, k, out_idx, out_dist, o, devices, ndev, st);
  cudaSetDevice(prev);
  return rc;
}

extern "C" int knn_join_partition_device(const float *q, int64_t m, const float *r, int64_t n,
                                         int32_t d, int32_t k, int32_t part, int32_t nparts,
                                         int32_t *out_idx, float *out_dist, int32_t *out_rows,
                                         int64_t *out_count, const knn_options *opt,
                                         knn_stats *st, void *stream) {
  error_buffer().clear();
  launch_counter() = 0;
  if (st) memset(st, 0, sizeof *st);
  if (out_count) *out_count = 0;
  knn_options o;
  int rc = check_options(opt, &o);
  if (rc == KNN_OK) rc = check_sizes(m, n, d, k);
  if (rc != KNN_OK) return rc;
  if (nparts <= 0 || part < 0 || part >= nparts || !out_count) {
    set_error("need 0 <= part < nparts and an out_count");
    return KNN_EINVAL;
  }
  if (m == 0) return KNN_OK;
  if (!q || !r || !out_idx || !out_dist || n == 0) {
    set_error(n == 0 ? "the partitioned join needs reference points" : "null pointer argument");
    return KNN_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool self = q == r && m == n;
  int Rs = o.sreps > 0 ? o.sreps : default_reps(n);
  if (Rs > n) Rs = (int)n;
  const int Rq = query_rep_count(o, m, d, k, self, Rs);
  const bool share = self && Rq == Rs;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      for (int i = 0; i < 3; i++)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  if (st)
    for (auto &e : ev) KNN_CUDA_TRY(cudaEventCreate(&e));
  if (st) KNN_CUDA_TRY(cudaEventRecord(ev[0], s));
  Arena ar(s);
  unsigned long long *ctr;
  KNN_TRY(ar.alloc(&ctr, kCtrCount));
  KNN_CUDA_TRY(cudaMemsetAsync(ctr, 0, kCtrCount * sizeof(unsigned long long), s));
  RefSide R;
  KNN_TRY(build_ref_side(ar, ar, r, n, d, Rs, o, false, reinterpret_cast<int *>(ctr + kCtrErr),
                         s, &R));
  QuerySide Q;
  KNN_TRY(build_query_side(R, share, q, m, k, o, ar, ctr, s, &Q));
  std::vector<int> cut;
  std::vector<int32_t> qoff;
  KNN_TRY(plan_parts(R, Q, nparts, ar, s, &cut, &qoff));
  if (st) KNN_CUDA_TRY(cudaEventRecord(ev[1], s));
  const int c0 = cut[part], c1 = cut[part + 1];
  const int64_t slot0 = qoff[c0], nslot = qoff[c1] - qoff[c0];
  KNN_TRY(search_clusters(R, Q, m, k, c0, c1, slot0, nslot, out_idx, out_dist, o, s, nullptr, ar,
                          ctr));
  if (st) KNN_CUDA_TRY(cudaEventRecord(ev[2], s));
  if (out_rows && nslot > 0)
    KNN_CUDA_TRY(cudaMemcpyAsync(out_rows, Q.qset.perm + slot0, sizeof(int32_t) * nslot,
                                 cudaMemcpyDeviceToDevice, s));
  *out_count = nslot;
  if (st) {
    KNN_TRY(read_stats(ctr, s, st));
    st->pairs_total = nslot * n;
    st->pairs_pruned = st->pairs_total - st->dist_evals;
    st->qreps_used = Q.Rq;
    st->sreps_used = R.Rs;
    st->kernels_launched = launch_counter();
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_build, ev[0], ev[1]));
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_search, ev[1], ev[2]));
    KNN_CUDA_TRY(cudaEventElapsedTime(&st->ms_total, ev[0], ev[2]));
  }
  return KNN_OK;
}
