/*
 * ref_shim.c -- TEST INFRASTRUCTURE ONLY.  LD_PRELOAD interposer used when the
 * reference's own CUDA program (oracle/_ref/knnjoin_ref, built by
 * oracle/build_ref.sh) is run as a checker and as the timing comparison.
 * It changes nothing in the reference's arithmetic; it makes its environment
 * deterministic and records its full result:
 *
 *  - cudaMalloc: the new block is zero-filled.  The reference reads device
 *    structures it never initialises (rep2q_static/rep2s_static are malloc'd
 *    on the host and copied over uninitialised: src/knnjoin.cu:1013-1014,
 *    246, 251 -- defect B3); with zeroed memory they start as the struct's
 *    own default member values (include/common8.h:42-48) intend.  Host malloc
 *    is zeroed by running with MALLOC_PERTURB_=255 (glibc fills new blocks with
 *    the complement of that byte).
 *  - cublasSgemm (legacy API): cublasInit() is called once before the first
 *    call -- the legacy API requires it and the reference never calls it --
 *    and the status after every call is logged to stderr.
 *  - cudaMemcpy device-to-host of exactly KNN_REF_DUMP_BYTES bytes (the final
 *    result copy, src/knnjoin.cu:1139-1141: query_nb*K IndexDist records) is
 *    also written to the file KNN_REF_DUMP_PATH.
 *
 * Build: gcc -O2 -fPIC -shared -o ref_shim.so ref_shim.c -ldl (build_ref.sh).
 * The reference binary must link the CUDA runtime dynamically (-cudart shared).
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

typedef int (*malloc_fn)(void **, size_t);
typedef int (*memset_fn)(void *, int, size_t);
typedef int (*memcpy_fn)(void *, const void *, size_t, int);
typedef void (*sgemm_fn)(char, char, int, int, int, float, const float *, int,
                         const float *, int, float, float *, int);
typedef int (*status_fn)(void);

static int g_inited = 0;

int cudaMalloc(void **p, size_t size) {
  static malloc_fn real = NULL;
  static memset_fn real_memset = NULL;
  if (!real) real = (malloc_fn)dlsym(RTLD_NEXT, "cudaMalloc");
  if (!real_memset) real_memset = (memset_fn)dlsym(RTLD_NEXT, "cudaMemset");
  int rc = real(p, size);
  if (rc == 0 && *p && size) real_memset(*p, 0, size);
  return rc;
}

int cudaMemcpy(void *dst, const void *src, size_t count, int kind) {
  static memcpy_fn real = NULL;
  if (!real) real = (memcpy_fn)dlsym(RTLD_NEXT, "cudaMemcpy");
  int rc = real(dst, src, count, kind);
  const char *want = getenv("KNN_REF_DUMP_BYTES");
  const char *path = getenv("KNN_REF_DUMP_PATH");
  if (rc == 0 && kind == 2 /* device to host */ && want && path &&
      (size_t)strtoull(want, NULL, 10) == count) {
    FILE *f = fopen(path, "wb");
    if (f) {
      fwrite(dst, 1, count, f);
      fclose(f);
    }
  }
  return rc;
}

void cublasSgemm(char ta, char tb, int m, int n, int k, float alpha, const float *A,
                 int lda, const float *B, int ldb, float beta, float *C, int ldc) {
  static sgemm_fn real = NULL;
  static status_fn get_error = NULL;
  if (!real) real = (sgemm_fn)dlsym(RTLD_NEXT, "cublasSgemm");
  if (!get_error) get_error = (status_fn)dlsym(RTLD_NEXT, "cublasGetError");
  if (!g_inited) {
    status_fn init = (status_fn)dlsym(RTLD_NEXT, "cublasInit");
    int st = init ? init() : -1;
    fprintf(stderr, "[ref_shim] cublasInit -> %d\n", st);
    g_inited = 1;
  }
  real(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  fprintf(stderr, "[ref_shim] cublasSgemm(%d,%d,%d) status %d\n", m, n, k,
          get_error ? get_error() : -1);
}
