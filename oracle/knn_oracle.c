/*
 * knn_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of knn_sweet's
 * exact kNN join, used as the checker by tests/, by __graft_entry__.smoke()
 * and by bench.py's CPU-baseline / reference arm.  Nothing in the product
 * (knn_sweet_b200/) links, loads or calls this file.
 *
 * It holds three things:
 *   1. glibc_rand: the glibc TYPE_3 additive-feedback generator behind
 *      srand()/rand() (the reference draws representative rows with it:
 *      src/knnjoin.cu:199-202, 226-229).  Restated from the published
 *      description of the algorithm (seed through the Park-Miller "minimal
 *      standard" multiplier 16807 mod 2^31-1, r[i] = r[i-3] + r[i-31] mod
 *      2^32, first 310 outputs discarded, output r >> 1).  Tests pin it
 *      against the C library's own rand().
 *   2. oracle_bruteforce_f64: FP64 brute force.  For each query the k
 *      smallest (squared distance, index) pairs over all reference rows,
 *      distances computed in double.  This is the correctness oracle.
 *   3. oracle_port_join: the reference's pruned method restated on the CPU
 *      (representative draw and spread score, nearest-representative
 *      assignment, members sorted by distance to the representative, the
 *      per-query-cluster k-th upper bound, the cluster-pair filter and the
 *      per-query banded triangle-inequality scan with a running k-th
 *      distance), with its defects B1 (missing reference-cluster radius,
 *      knnjoin.cu:391, 515) and B2 (upper bound replacing every tied maximum,
 *      knnjoin.cu:486-489) fixed so that the result is exact.  OpenMP over
 *      queries; it is the CPU baseline timed beside the GPU.
 *
 * Tie rule everywhere: ascending squared distance, then ascending index.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* 1. glibc rand() restatement                                                */
/* ------------------------------------------------------------------------- */

typedef struct glibc_rand_state {
  int32_t r[34];
  int32_t pos; /* ring position: r holds the last 34 values */
  uint32_t ring[34];
} glibc_rand_state;

/* srand(seed): seed 0 behaves like 1 (glibc maps a zero seed to 1). */
void glibc_srand(glibc_rand_state *s, uint32_t seed) {
  int64_t r[344 + 34];
  int i;
  if (seed == 0) seed = 1;
  r[0] = (int32_t)seed;
  for (i = 1; i < 31; i++) {
    /* r[i] = 16807 * r[i-1] mod (2^31 - 1), kept in signed 32-bit range */
    int64_t v = (16807LL * r[i - 1]) % 2147483647LL;
    if (v < 0) v += 2147483647LL;
    r[i] = v;
  }
  for (i = 31; i < 34; i++) r[i] = r[i - 31];
  for (i = 34; i < 344; i++)
    r[i] = (int64_t)(uint32_t)((uint32_t)r[i - 31] + (uint32_t)r[i - 3]);
  for (i = 0; i < 34; i++) s->ring[i] = (uint32_t)r[344 - 34 + i];
  s->pos = 0; /* ring[pos] is the oldest value, r[i-34] */
}

int32_t glibc_rand(glibc_rand_state *s) {
  /* next = r[i-31] + r[i-3]; ring holds r[i-34 .. i-1] with r[i-34] at pos */
  uint32_t a = s->ring[(s->pos + 3) % 34];  /* r[i-31] */
  uint32_t b = s->ring[(s->pos + 31) % 34]; /* r[i-3]  */
  uint32_t v = a + b;
  s->ring[s->pos] = v;
  s->pos = (s->pos + 1) % 34;
  return (int32_t)(v >> 1);
}

/* Fill out[0..count) with successive rand() values after srand(seed). */
void oracle_glibc_rand_seq(uint32_t seed, int64_t count, int32_t *out) {
  glibc_rand_state s;
  int64_t i;
  glibc_srand(&s, seed);
  for (i = 0; i < count; i++) out[i] = glibc_rand(&s);
}

/* ------------------------------------------------------------------------- */
/* Shared helpers                                                             */
/* ------------------------------------------------------------------------- */

/* FP32 squared distance in dimension order with fused multiply-add, the form
 * the device code uses (Edistance_128 accumulates dimension by dimension:
 * include/common8.h:153-175; nvcc contracts `distance += tmp*tmp` to an fma). */
static inline float dist2_f32(const float *a, const float *b, int d) {
  float acc = 0.0f;
  for (int i = 0; i < d; i++) {
    float t = a[i] - b[i];
    acc = fmaf(t, t, acc);
  }
  return acc;
}

static inline double dist2_f64(const float *a, const float *b, int d) {
  double acc = 0.0;
  for (int i = 0; i < d; i++) {
    double t = (double)a[i] - (double)b[i];
    acc += t * t;
  }
  return acc;
}

typedef struct {
  double key;
  int32_t idx;
} kd64;

/* max-heap on (key, idx) */
static inline int kd64_less(kd64 a, kd64 b) {
  return a.key < b.key || (a.key == b.key && a.idx < b.idx);
}

static void heap64_sift_down(kd64 *h, int n, int i) {
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < n && kd64_less(h[m], h[l])) m = l;
    if (r < n && kd64_less(h[m], h[r])) m = r;
    if (m == i) return;
    kd64 t = h[i];
    h[i] = h[m];
    h[m] = t;
    i = m;
  }
}

static void heap64_sift_up(kd64 *h, int i) {
  while (i > 0) {
    int p = (i - 1) / 2;
    if (!kd64_less(h[p], h[i])) return;
    kd64 t = h[i];
    h[i] = h[p];
    h[p] = t;
    i = p;
  }
}

static int cmp_kd64(const void *a, const void *b) {
  kd64 x = *(const kd64 *)a, y = *(const kd64 *)b;
  if (kd64_less(x, y)) return -1;
  if (kd64_less(y, x)) return 1;
  return 0;
}

static int resolve_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* 2. FP64 brute force                                                        */
/* ------------------------------------------------------------------------- */

/*
 * For each of the `nq` query rows listed in qrows (or rows 0..m-1 when qrows
 * is NULL, nq = m): the k nearest reference rows, ascending (d^2, index), in
 * FP64.  out_idx / out_dist are nq x k; missing slots (k > n) hold -1 / +inf.
 * out_dist holds the Euclidean distance sqrt(d^2).
 */
int oracle_bruteforce_f64(const float *q, int64_t m, const float *r, int64_t n,
                          int32_t d, int32_t k, const int64_t *qrows,
                          int64_t nq, int32_t *out_idx, double *out_dist,
                          int nthreads) {
  if (!q || !r || d <= 0 || k <= 0 || n < 0 || m < 0) return -1;
  if (!qrows) nq = m;
  int nt = resolve_threads(nthreads);
  int64_t t;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
  for (t = 0; t < nq; t++) {
    int64_t qi = qrows ? qrows[t] : t;
    const float *qp = q + qi * (int64_t)d;
    kd64 *heap = (kd64 *)malloc(sizeof(kd64) * (size_t)k);
    int hn = 0;
    for (int64_t j = 0; j < n; j++) {
      kd64 c;
      c.key = dist2_f64(qp, r + j * (int64_t)d, d);
      c.idx = (int32_t)j;
      if (hn < k) {
        heap[hn] = c;
        heap64_sift_up(heap, hn);
        hn++;
      } else if (kd64_less(c, heap[0])) {
        heap[0] = c;
        heap64_sift_down(heap, hn, 0);
      }
    }
    qsort(heap, (size_t)hn, sizeof(kd64), cmp_kd64);
    for (int j = 0; j < k; j++) {
      if (j < hn) {
        out_idx[t * k + j] = heap[j].idx;
        out_dist[t * k + j] = sqrt(heap[j].key);
      } else {
        out_idx[t * k + j] = -1;
        out_dist[t * k + j] = INFINITY;
      }
    }
    free(heap);
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* 3. CPU restatement of the reference's pruned join                          */
/* ------------------------------------------------------------------------- */

/*
 * Representative draw (src/knnjoin.cu:195-239, kernels 125-154): after
 * srand(seed), `trials` rows of `reps` indices rand() % n; each trial is
 * scored by the int32 (wrapping) sum over all ordered pairs (i, j), i == j
 * included, of (int) of the FP32 distance; the first trial whose score,
 * compared as float, beats the running best (starting at 0.0f) wins.
 * Writes the winning trial's row indices to out_rows[0..reps).  Returns the
 * winning trial.
 */
int oracle_select_reps(const float *pts, int64_t n, int32_t d, int32_t reps,
                       uint32_t seed, int32_t trials, int32_t *out_rows) {
  glibc_rand_state s;
  glibc_srand(&s, seed);
  int32_t *cand = (int32_t *)malloc(sizeof(int32_t) * (size_t)trials * reps);
  for (int t = 0; t < trials; t++)
    for (int i = 0; i < reps; i++)
      cand[t * reps + i] = (int32_t)(glibc_rand(&s) % (int32_t)n);
  float best = 0.0f;
  int best_t = 0;
  for (int t = 0; t < trials; t++) {
    uint32_t sum = 0;
    for (int i = 0; i < reps; i++) {
      const float *a = pts + (int64_t)cand[t * reps + i] * d;
      for (int j = 0; j < reps; j++) {
        const float *b = pts + (int64_t)cand[t * reps + j] * d;
        sum += (uint32_t)(int32_t)sqrtf(dist2_f32(a, b, d));
      }
    }
    if (best < (float)(int32_t)sum) {
      best = (float)(int32_t)sum;
      best_t = t;
    }
  }
  memcpy(out_rows, cand + best_t * reps, sizeof(int32_t) * reps);
  free(cand);
  return best_t;
}

typedef struct {
  float dist;
  int32_t idx;
} fd32;

static int cmp_fd32(const void *a, const void *b) {
  fd32 x = *(const fd32 *)a, y = *(const fd32 *)b;
  if (x.dist < y.dist) return -1;
  if (x.dist > y.dist) return 1;
  return (x.idx > y.idx) - (x.idx < y.idx);
}

/* Nearest representative (lowest representative index on ties), as
 * findQCluster / findTCluster (src/knnjoin.cu:64-97). */
static void assign_points(const float *pts, int64_t n, int32_t d,
                          const float *reps, int32_t nrep, int32_t *cl,
                          float *dr, int nt) {
  int64_t i;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (i = 0; i < n; i++) {
    float best = FLT_MAX;
    int bi = -1;
    for (int j = 0; j < nrep; j++) {
      float v = dist2_f32(pts + i * d, reps + (int64_t)j * d, d);
      if (v < best) {
        best = v;
        bi = j;
      }
    }
    cl[i] = bi;
    dr[i] = sqrtf(best);
  }
}

/* Relative slack covering FP32 rounding of the distances entering a bound. */
static inline float port_tol(int32_t d) {
  return (float)(4 * d + 16) * 5.9604645e-8f;
}

typedef struct oracle_port_stats {
  int64_t dist_evals;
  int64_t clusters_visited;
  int64_t clusters_pruned;
  int32_t qreps_trial;
  int32_t sreps_trial;
  double build_seconds; /* representatives .. cluster filter */
  double scan_seconds;  /* per-query scan of the requested rows */
} oracle_port_stats;

static double wall_seconds(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return (double)clock() / CLOCKS_PER_SEC;
#endif
}

/*
 * The reference's pruned join restated on the CPU.  Queries processed are
 * qrows[0..nq) (or all m when qrows is NULL); out_idx / out_dist are nq x k
 * (float Euclidean distances, ascending (d^2, index)).  The index build
 * (representatives, assignment, sorting, bounds, filter) always covers the
 * full sets.  Returns 0 on success.
 */
int oracle_port_join(const float *q, int64_t m, const float *r, int64_t n,
                     int32_t d, int32_t k, int32_t qreps, int32_t sreps,
                     uint32_t seed, int32_t trials, const int64_t *qrows,
                     int64_t nq, int32_t *out_idx, float *out_dist,
                     oracle_port_stats *st, int nthreads) {
  if (!q || !r || d <= 0 || k <= 0 || n <= 0 || m <= 0) return -1;
  if (qreps > m) qreps = (int32_t)m;
  if (sreps > n) sreps = (int32_t)n;
  if (!qrows) nq = m;
  int nt = resolve_threads(nthreads);
  const float tol = port_tol(d);
  double t_start = wall_seconds();

  /* representatives (knnjoin.cu:195-239) */
  int32_t *qrow = (int32_t *)malloc(sizeof(int32_t) * qreps);
  int32_t *srow = (int32_t *)malloc(sizeof(int32_t) * sreps);
  int qt = oracle_select_reps(q, m, d, qreps, seed, trials, qrow);
  int stt = oracle_select_reps(r, n, d, sreps, seed, trials, srow);
  float *qrep = (float *)malloc(sizeof(float) * (size_t)qreps * d);
  float *srep = (float *)malloc(sizeof(float) * (size_t)sreps * d);
  for (int i = 0; i < qreps; i++)
    memcpy(qrep + (int64_t)i * d, q + (int64_t)qrow[i] * d, sizeof(float) * d);
  for (int i = 0; i < sreps; i++)
    memcpy(srep + (int64_t)i * d, r + (int64_t)srow[i] * d, sizeof(float) * d);

  /* assignment (knnjoin.cu:275-295, 331-342) */
  int32_t *qcl = (int32_t *)malloc(sizeof(int32_t) * m);
  float *qdr = (float *)malloc(sizeof(float) * m);
  int32_t *scl = (int32_t *)malloc(sizeof(int32_t) * n);
  float *sdr = (float *)malloc(sizeof(float) * n);
  assign_points(q, m, d, qrep, qreps, qcl, qdr, nt);
  assign_points(r, n, d, srep, sreps, scl, sdr, nt);

  /* query radius maxquery (knnjoin.cu:78) */
  float *qrad = (float *)calloc((size_t)qreps, sizeof(float));
  for (int64_t i = 0; i < m; i++)
    if (qdr[i] > qrad[qcl[i]]) qrad[qcl[i]] = qdr[i];

  /* members of every reference cluster sorted by distance to the
   * representative (fillTMembers + host sort, knnjoin.cu:352, 382-399) */
  int64_t *off = (int64_t *)calloc((size_t)sreps + 1, sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) off[scl[i] + 1]++;
  for (int i = 0; i < sreps; i++) off[i + 1] += off[i];
  fd32 *mem = (fd32 *)malloc(sizeof(fd32) * n);
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * sreps);
  for (int i = 0; i < sreps; i++) fill[i] = off[i];
  for (int64_t i = 0; i < n; i++) {
    fd32 e = {sdr[i], (int32_t)i};
    mem[fill[scl[i]]++] = e;
  }
  free(fill);
  int i32;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (i32 = 0; i32 < sreps; i32++)
    qsort(mem + off[i32], (size_t)(off[i32 + 1] - off[i32]), sizeof(fd32),
          cmp_fd32);
  /* B1 fixed: the cluster radius is the largest member distance. */
  float *srad = (float *)calloc((size_t)sreps, sizeof(float));
  for (int i = 0; i < sreps; i++)
    srad[i] = off[i + 1] > off[i] ? mem[off[i + 1] - 1].dist : 0.0f;

  /* representative-to-representative distances */
  float *drr = (float *)malloc(sizeof(float) * (size_t)qreps * sreps);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (i32 = 0; i32 < qreps; i32++)
    for (int j = 0; j < sreps; j++)
      drr[(int64_t)i32 * sreps + j] =
          sqrtf(dist2_f32(qrep + (int64_t)i32 * d, srep + (int64_t)j * d, d));

  /* per query cluster: k-th smallest of rq + d(Rq,Rs) + d(s,Rs) over all
   * reference points (RepsUpperBound, knnjoin.cu:459-504; B2 fixed by an
   * exact selection), widened by the rounding slack -> theta0.  Then the
   * cluster filter (FilterReps, knnjoin.cu:506-525) with the true radius,
   * and the surviving list sorted by d(Rq,Rs) (knnjoin.cu:1080-1091). */
  float *theta0 = (float *)malloc(sizeof(float) * qreps);
  int32_t *rl = (int32_t *)malloc(sizeof(int32_t) * (size_t)qreps * sreps);
  int32_t *rlen = (int32_t *)calloc((size_t)qreps, sizeof(int32_t));
  int64_t kk = k < n ? k : n;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (i32 = 0; i32 < qreps; i32++) {
    float rq = qrad[i32];
    /* k smallest bound values: per cluster the first min(k, size) members */
    int64_t cap = 0;
    for (int j = 0; j < sreps; j++) {
      int64_t sz = off[j + 1] - off[j];
      cap += sz < kk ? sz : kk;
    }
    float *vals = (float *)malloc(sizeof(float) * (size_t)cap);
    int64_t nv = 0;
    for (int j = 0; j < sreps; j++) {
      float base = rq + drr[(int64_t)i32 * sreps + j];
      int64_t sz = off[j + 1] - off[j];
      int64_t lim = sz < kk ? sz : kk;
      for (int64_t t = 0; t < lim; t++) vals[nv++] = base + mem[off[j] + t].dist;
    }
    /* k-th smallest by partial selection (quickselect) */
    int64_t want = kk - 1, lo = 0, hi = nv - 1;
    while (lo < hi) {
      float piv = vals[(lo + hi) / 2];
      int64_t a = lo, b = hi;
      while (a <= b) {
        while (vals[a] < piv) a++;
        while (vals[b] > piv) b--;
        if (a <= b) {
          float t = vals[a];
          vals[a] = vals[b];
          vals[b] = t;
          a++;
          b--;
        }
      }
      if (want <= b) hi = b;
      else if (want >= a) lo = a;
      else break;
    }
    float kth = vals[want];
    free(vals);
    float th = kth * (1.0f + 4.0f * tol) + FLT_MIN;
    theta0[i32] = th;
    /* filter and sort by d(Rq,Rs) then index */
    fd32 *tmp = (fd32 *)malloc(sizeof(fd32) * sreps);
    int cnt = 0;
    for (int j = 0; j < sreps; j++) {
      if (off[j + 1] == off[j]) continue;
      float dd = drr[(int64_t)i32 * sreps + j];
      float lb = dd - rq - srad[j];
      if (lb > th + tol * (dd + rq + srad[j] + th)) continue;
      fd32 e = {dd, j};
      tmp[cnt++] = e;
    }
    qsort(tmp, (size_t)cnt, sizeof(fd32), cmp_fd32);
    for (int j = 0; j < cnt; j++) rl[(int64_t)i32 * sreps + j] = tmp[j].idx;
    rlen[i32] = cnt;
    free(tmp);
  }

  /* per-query scan (KNNQuery_base, knnjoin.cu:762-858): over the surviving
   * clusters nearest first; inside a cluster only members whose distance to
   * the representative lies within theta of d(q,Rs) can be closer than the
   * running k-th neighbour; insertion into a sorted list of k. */
  double t_built = wall_seconds();
  int64_t evals = 0, visited = 0, pruned = 0;
  int64_t t;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt) \
    reduction(+ : evals, visited, pruned)
  for (t = 0; t < nq; t++) {
    int64_t qi = qrows ? qrows[t] : t;
    const float *qp = q + qi * d;
    int c = qcl[qi];
    /* keys: (d^2, idx) ordered; the list holds the best `cnt` so far */
    float *ld = (float *)malloc(sizeof(float) * (size_t)k);
    int32_t *li = (int32_t *)malloc(sizeof(int32_t) * (size_t)k);
    int cnt = 0;
    float th_d2 = theta0[c] * theta0[c];
    float th = theta0[c];
    for (int a = 0; a < rlen[c]; a++) {
      int rs = rl[(int64_t)c * sreps + a];
      float D = sqrtf(dist2_f32(qp, srep + (int64_t)rs * d, d));
      float slack = tol * (2.0f * D + 2.0f * th);
      if (D - srad[rs] > th + slack || D + th + slack < mem[off[rs]].dist) {
        pruned++;
        continue;
      }
      visited++;
      /* band [D - th, D + th] in the ascending member distances */
      float lo_v = D - th - slack;
      int64_t lo = off[rs], hi = off[rs + 1];
      while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (mem[mid].dist < lo_v) lo = mid + 1;
        else hi = mid;
      }
      for (int64_t p = lo; p < off[rs + 1]; p++) {
        slack = tol * (2.0f * D + 2.0f * th);
        if (mem[p].dist > D + th + slack) break;
        int32_t si = mem[p].idx;
        float v = dist2_f32(qp, r + (int64_t)si * d, d);
        evals++;
        /* enters iff (v, si) < (th_d2, last idx) once full, v <= th_d2 while
         * filling (theta0 admits ties) */
        if (cnt == k) {
          if (v > ld[k - 1] || (v == ld[k - 1] && si > li[k - 1])) continue;
        } else if (v > th_d2) {
          continue;
        }
        int pos = cnt < k ? cnt : k - 1;
        while (pos > 0 && (ld[pos - 1] > v || (ld[pos - 1] == v && li[pos - 1] > si))) {
          if (pos < k) {
            ld[pos] = ld[pos - 1];
            li[pos] = li[pos - 1];
          }
          pos--;
        }
        ld[pos] = v;
        li[pos] = si;
        if (cnt < k) cnt++;
        if (cnt == k) {
          th_d2 = ld[k - 1];
          th = sqrtf(th_d2);
        }
      }
    }
    for (int j = 0; j < k; j++) {
      if (j < cnt) {
        out_idx[t * k + j] = li[j];
        out_dist[t * k + j] = sqrtf(ld[j]);
      } else {
        out_idx[t * k + j] = -1;
        out_dist[t * k + j] = INFINITY;
      }
    }
    free(ld);
    free(li);
  }
  double t_done = wall_seconds();
  if (st) {
    st->build_seconds = t_built - t_start;
    st->scan_seconds = t_done - t_built;
    st->dist_evals = evals;
    st->clusters_visited = visited;
    st->clusters_pruned = pruned;
    st->qreps_trial = qt;
    st->sreps_trial = stt;
  }
  free(qrow); free(srow); free(qrep); free(srep); free(qcl); free(qdr);
  free(scl); free(sdr); free(qrad); free(off); free(mem); free(srad);
  free(drr); free(theta0); free(rl); free(rlen);
  return 0;
}

int oracle_num_threads(void) { return resolve_threads(0); }
