/*
 * zheevr_fwd.c -- LAPACK zheevr_ forwarder for the oracle build.
 *
 * TEST INFRASTRUCTURE ONLY.  K-Litho-TCC/klitho_tcc.cpp:292-298 declares
 * zheevr_ with the Fortran LP64 ABI and calls it at :327 and :340.  This image
 * has no system LAPACK, so this file supplies that symbol by forwarding to the
 * `scipy_zheevr_` export of the OpenBLAS 0.3.30 build that ships with scipy
 * (scipy.libs/libscipy_openblas-*.so).  The library is opened at first use,
 * from $KLITHO_OPENBLAS or the path fixed at build time.  BLAS threading is
 * pinned to one thread so results are reproducible run to run.
 *
 * Never linked into the GPU product: the product's eigen-solver is its own
 * subspace iteration on the GPU.
 */
#include <dlfcn.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#ifndef KL_OPENBLAS_PATH
#define KL_OPENBLAS_PATH "libscipy_openblas.so"
#endif

typedef void (*zheevr_fn)(const char*, const char*, const char*, int*, void*, int*, double*,
                          double*, int*, int*, double*, int*, double*, void*, int*, int*, void*,
                          int*, double*, int*, int*, int*, int*, size_t, size_t, size_t);
typedef void (*setthreads_fn)(int);

static zheevr_fn resolve(void) {
  static zheevr_fn fn = NULL;
  if (fn) return fn;
  const char* path = getenv("KLITHO_OPENBLAS");
  if (!path || !*path) path = KL_OPENBLAS_PATH;
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    fprintf(stderr, "zheevr_fwd: cannot open %s: %s\n", path, dlerror());
    abort();
  }
  setthreads_fn st = (setthreads_fn)dlsym(h, "scipy_openblas_set_num_threads");
  if (st) st(1);
  fn = (zheevr_fn)dlsym(h, "scipy_zheevr_");
  if (!fn) {
    fprintf(stderr, "zheevr_fwd: scipy_zheevr_ not found in %s\n", path);
    abort();
  }
  return fn;
}

/* Same argument list as the reference's prototype (klitho_tcc.cpp:294-297);
 * the three Fortran hidden character lengths are supplied here. */
void zheevr_(const char* jobz, const char* range, const char* uplo, int* n, void* a, int* lda,
             double* vl, double* vu, int* il, int* iu, double* abstol, int* m, double* w, void* z,
             int* ldz, int* isuppz, void* work, int* lwork, double* rwork, int* lrwork, int* iwork,
             int* liwork, int* info) {
  resolve()(jobz, range, uplo, n, a, lda, vl, vu, il, iu, abstol, m, w, z, ldz, isuppz, work,
            lwork, rwork, lrwork, iwork, liwork, info, 1, 1, 1);
}
