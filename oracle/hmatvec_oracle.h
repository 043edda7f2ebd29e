/* CPU restatement of the reference H-matrix products -- TEST INFRASTRUCTURE.
 *
 * Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark may call this code; it is the checker, never the product.
 *
 * Block storage follows the reference: every block is compact column-major
 * (il::Array2D, il/il/container/2d/Array2D.h:840, ld = rows), a low-rank block
 * is A (m x r) and B (r x n) with y += A (B x)
 * (src/hmat/hmatrix/hmat.cc:510-527, LowRank.h:18-24).  Pattern rows are in
 * collocation-point units as in HPattern (src/hmat/hmatrix/h_pattern.h:21-33);
 * scalar rows are point * dof + component.
 */
#ifndef HMATVEC_ORACLE_H
#define HMATVEC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t dof;              /* dofs per collocation point */
  int32_t pad_;
  int64_t n_rows, n_cols;   /* scalar sizes (size_[0], size_[1]) */
  int64_t n_fr, n_lr;       /* block counts */
  const int64_t *fr;        /* n_fr x 4: i0, j0, iend, jend (points) */
  const int64_t *lr;        /* n_lr x 5: i0, j0, iend, jend, r (scalar columns of A) */
  const double *fr_data;    /* FR blocks back to back, column-major */
  const double *lr_data;    /* per LR block: A (m x r) then B (r x n), column-major */
  const int64_t *perm0;     /* n_rows/dof, row permutation (permutation_0_) */
  const int64_t *perm1;     /* n_cols/dof, column permutation (permutation_1_) */
} oracle_hmat;

/* y = H x in the permuted ordering (Hmat::matvec, hmat.cc:472-537). */
int oracle_matvec_perm(const oracle_hmat *h, const double *x, double *y, int nthreads);
/* y = H x in the original ordering (Hmat::matvecOriginal, hmat.cc:572-635). */
int oracle_matvec(const oracle_hmat *h, const double *x, double *y, int nthreads);
/* y = H^T x, permuted / original ordering (no reference counterpart; applies
 * each block's transpose: FR A^T, LR B^T (A^T x)). */
int oracle_rmatvec_perm(const oracle_hmat *h, const double *x, double *y, int nthreads);
int oracle_rmatvec(const oracle_hmat *h, const double *x, double *y, int nthreads);
/* Y = H X for k right-hand sides, X is n_cols x k and Y is n_rows x k, both
 * column-major, original ordering (no reference counterpart). */
int oracle_matmat(const oracle_hmat *h, const double *X, double *Y, int64_t k, int nthreads);
/* Diagonal in the original ordering (Hmat::diagonalOriginal, hmat.cc:240-285). */
int oracle_diagonal(const oracle_hmat *h, double *d);
/* Total stored entries (Hmat::nbOfEntries, hmat.cc:300-313). */
int64_t oracle_entries(const oracle_hmat *h);

#ifdef __cplusplus
}
#endif
#endif
