// CBLAS adapter for compiling the reference's CPU sources: the two routines
// they call (cblas_dgemm, cblas_dsyr2k) forwarded to the 64-bit-integer
// OpenBLAS build that ships with numpy (symbols scipy_cblas_*64_).  Test
// infrastructure only.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };

void scipy_cblas_dgemm64_(int order, int ta, int tb, long long m, long long n, long long k, double alpha,
                          const double *a, long long lda, const double *b, long long ldb, double beta, double *c,
                          long long ldc);
void scipy_cblas_dsyr2k64_(int order, int uplo, int trans, long long n, long long k, double alpha, const double *a,
                           long long lda, const double *b, long long ldb, double beta, double *c, long long ldc);

static inline void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n,
                               int k, double alpha, const double *a, int lda, const double *b, int ldb, double beta,
                               double *c, int ldc) {
  scipy_cblas_dgemm64_(order, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
static inline void cblas_dsyr2k(enum CBLAS_ORDER order, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE trans, int n, int k,
                                double alpha, const double *a, int lda, const double *b, int ldb, double beta, double *c,
                                int ldc) {
  scipy_cblas_dsyr2k64_(order, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
#ifdef __cplusplus
}
#endif
