/* Prototype-only CBLAS header.
 *
 * The reference's IL headers include <cblas.h> when built with IL_OPENBLAS
 * (il/il/linearAlgebra/dense/blas/blas_config.h).  This image ships an
 * OpenBLAS shared library (inside the opencv wheel) but no development
 * headers, so this file declares the standard CBLAS enums and the routines
 * those headers reference, following the netlib CBLAS interface.
 * The symbols themselves come from the OpenBLAS library at link time.
 */
#ifndef BW_SHIM_CBLAS_H
#define BW_SHIM_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum CBLAS_TRANSPOSE {
  CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113, CblasConjNoTrans = 114
} CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

typedef struct { float real, imag; } openblas_complex_float;
typedef struct { double real, imag; } openblas_complex_double;

/* level 1 */
void cblas_saxpy(int n, float alpha, const float *x, int incx, float *y, int incy);
void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy);
void cblas_caxpy(int n, const void *alpha, const void *x, int incx, void *y, int incy);
void cblas_zaxpy(int n, const void *alpha, const void *x, int incx, void *y, int incy);
void cblas_saxpby(int n, float alpha, const float *x, int incx, float beta, float *y, int incy);
void cblas_daxpby(int n, double alpha, const double *x, int incx, double beta, double *y, int incy);
void cblas_caxpby(int n, const void *alpha, const void *x, int incx, const void *beta, void *y, int incy);
void cblas_zaxpby(int n, const void *alpha, const void *x, int incx, const void *beta, void *y, int incy);
float cblas_sdot(int n, const float *x, int incx, const float *y, int incy);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
void cblas_cdotu_sub(int n, const void *x, int incx, const void *y, int incy, void *dotu);
void cblas_cdotc_sub(int n, const void *x, int incx, const void *y, int incy, void *dotc);
void cblas_zdotu_sub(int n, const void *x, int incx, const void *y, int incy, void *dotu);
void cblas_zdotc_sub(int n, const void *x, int incx, const void *y, int incy, void *dotc);

/* level 2 */
void cblas_sgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, float alpha,
                 const float *a, int lda, const float *x, int incx, float beta, float *y, int incy);
void cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, double alpha,
                 const double *a, int lda, const double *x, int incx, double beta, double *y, int incy);
void cblas_cgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, const void *alpha,
                 const void *a, int lda, const void *x, int incx, const void *beta, void *y, int incy);
void cblas_zgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, const void *alpha,
                 const void *a, int lda, const void *x, int incx, const void *beta, void *y, int incy);

/* level 3 */
void cblas_sgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k,
                 float alpha, const float *a, int lda, const float *b, int ldb, float beta, float *c, int ldc);
void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k,
                 double alpha, const double *a, int lda, const double *b, int ldb, double beta, double *c, int ldc);
void cblas_cgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k,
                 const void *alpha, const void *a, int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
void cblas_zgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k,
                 const void *alpha, const void *a, int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
void cblas_dtrsm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo, CBLAS_TRANSPOSE ta, CBLAS_DIAG diag,
                 int m, int n, double alpha, const double *a, int lda, double *b, int ldb);
void cblas_ztrsm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo, CBLAS_TRANSPOSE ta, CBLAS_DIAG diag,
                 int m, int n, const void *alpha, const void *a, int lda, void *b, int ldb);

/* OpenBLAS extension: thread count of the BLAS itself. */
void openblas_set_num_threads(int num_threads);

#ifdef __cplusplus
}
#endif

#endif /* BW_SHIM_CBLAS_H */
