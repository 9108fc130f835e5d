/* LAPACK/BLAS name forwarders: TEST INFRASTRUCTURE ONLY.
 *
 * The reference's subspace eigensolver calls Fortran LAPACK `dsyev_`
 * (framework/hp_numeric.h:500-520) and its GEMM helper calls `dgemm_`.  This image has no
 * system LAPACK; SciPy's bundled OpenBLAS exports the same routines under a `scipy_` prefix.
 * These thin wrappers forward the reference's calls to it so the reference compiles and
 * links unchanged.  Only the reference build under oracle/_ref links this file. */
#include <stddef.h>

extern void scipy_dsyev_(char *, char *, int *, double *, int *, double *, double *, int *, int *,
                         size_t, size_t);
extern void scipy_dgemm_(char *, char *, int *, int *, int *, double *, double *, int *, double *,
                         int *, double *, double *, int *, size_t, size_t);
extern void scipy_sgemm_(char *, char *, int *, int *, int *, float *, float *, int *, float *,
                         int *, float *, float *, int *, size_t, size_t);

void dsyev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w, double *work,
            int *lwork, int *info) {
  scipy_dsyev_(jobz, uplo, n, a, lda, w, work, lwork, info, 1, 1);
}

void dgemm_(char *ta, char *tb, int *m, int *n, int *k, double *alpha, double *a, int *lda,
            double *b, int *ldb, double *beta, double *c, int *ldc) {
  scipy_dgemm_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}

void sgemm_(char *ta, char *tb, int *m, int *n, int *k, float *alpha, float *a, int *lda,
            float *b, int *ldb, float *beta, float *c, int *ldc) {
  scipy_sgemm_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}
