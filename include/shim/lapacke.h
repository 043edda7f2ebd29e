/* Prototype-only LAPACKE header.
 *
 * Declares the standard LAPACKE C interface for the routines that the
 * reference's IL headers (il/il/linearAlgebra/dense/...) call when built with
 * IL_OPENBLAS.  Symbols are resolved against the OpenBLAS shared library.
 */
#ifndef BW_SHIM_LAPACKE_H
#define BW_SHIM_LAPACKE_H

#include <complex>

#define lapack_int int
#define lapack_logical int
#define lapack_complex_float std::complex<float>
#define lapack_complex_double std::complex<double>
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

extern "C" {
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda, lapack_int *ipiv);
lapack_int LAPACKE_zgetrf(int layout, lapack_int m, lapack_int n, lapack_complex_double *a, lapack_int lda,
                          lapack_int *ipiv);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double *a, lapack_int lda, const lapack_int *ipiv);
lapack_int LAPACKE_zgetri(int layout, lapack_int n, lapack_complex_double *a, lapack_int lda,
                          const lapack_int *ipiv);
lapack_int LAPACKE_dgetrs(int layout, char trans, lapack_int n, lapack_int nrhs, const double *a, lapack_int lda,
                          const lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a, lapack_int lda, lapack_int *ipiv,
                         double *b, lapack_int ldb);
lapack_int LAPACKE_dgecon(int layout, char norm, lapack_int n, const double *a, lapack_int lda, double anorm,
                          double *rcond);
lapack_int LAPACKE_dgbsv(int layout, lapack_int n, lapack_int kl, lapack_int ku, lapack_int nrhs, double *ab,
                         lapack_int ldab, lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dgtsv(int layout, lapack_int n, lapack_int nrhs, double *dl, double *d, double *du, double *b,
                         lapack_int ldb);
lapack_int LAPACKE_dgebrd(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda, double *d, double *e,
                          double *tauq, double *taup);
lapack_int LAPACKE_zgebrd(int layout, lapack_int m, lapack_int n, lapack_complex_double *a, lapack_int lda,
                          double *d, double *e, lapack_complex_double *tauq, lapack_complex_double *taup);
lapack_int LAPACKE_dbdsqr(int layout, char uplo, lapack_int n, lapack_int ncvt, lapack_int nru, lapack_int ncc,
                          double *d, double *e, double *vt, lapack_int ldvt, double *u, lapack_int ldu, double *c,
                          lapack_int ldc);
lapack_int LAPACKE_zbdsqr(int layout, char uplo, lapack_int n, lapack_int ncvt, lapack_int nru, lapack_int ncc,
                          double *d, double *e, lapack_complex_double *vt, lapack_int ldvt,
                          lapack_complex_double *u, lapack_int ldu, lapack_complex_double *c, lapack_int ldc);
lapack_int LAPACKE_dlaswp(int layout, lapack_int n, double *a, lapack_int lda, lapack_int k1, lapack_int k2,
                          const lapack_int *ipiv, lapack_int incx);
lapack_int LAPACKE_zlaswp(int layout, lapack_int n, lapack_complex_double *a, lapack_int lda, lapack_int k1,
                          lapack_int k2, const lapack_int *ipiv, lapack_int incx);
lapack_int LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda, double *tau);
lapack_int LAPACKE_zgeqrf(int layout, lapack_int m, lapack_int n, lapack_complex_double *a, lapack_int lda,
                          lapack_complex_double *tau);
lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double *a, lapack_int lda,
                          double *s, double *u, lapack_int ldu, double *vt, lapack_int ldvt, double *superb);
lapack_int LAPACKE_dpotrf(int layout, char uplo, lapack_int n, double *a, lapack_int lda);
lapack_int LAPACKE_dpotrs(int layout, char uplo, lapack_int n, lapack_int nrhs, const double *a, lapack_int lda,
                          double *b, lapack_int ldb);
lapack_int LAPACKE_dpotri(int layout, char uplo, lapack_int n, double *a, lapack_int lda);
lapack_int LAPACKE_dpocon(int layout, char uplo, lapack_int n, const double *a, lapack_int lda, double anorm,
                          double *rcond);
lapack_int LAPACKE_dpptrf(int layout, char uplo, lapack_int n, double *ap);
lapack_int LAPACKE_dgehrd(int layout, lapack_int n, lapack_int ilo, lapack_int ihi, double *a, lapack_int lda,
                          double *tau);
lapack_int LAPACKE_dhseqr(int layout, char job, char compz, lapack_int n, lapack_int ilo, lapack_int ihi, double *h,
                          lapack_int ldh, double *wr, double *wi, double *z, lapack_int ldz);
}

#endif /* BW_SHIM_LAPACKE_H */
