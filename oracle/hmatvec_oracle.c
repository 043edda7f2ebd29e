/* CPU restatement of the reference H-matrix products -- TEST INFRASTRUCTURE.
 *
 * The checker for the CUDA backend: only tests/, the smoke check and the
 * CPU-baseline leg of bench.py call it.  Every routine follows the reference
 * routine cited above it; the arithmetic is plain double-precision loops in
 * the order a column-major dgemv would use.
 */
#include "hmatvec_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

static int64_t fr_m(const oracle_hmat *h, int64_t k) { return (h->fr[4 * k + 2] - h->fr[4 * k + 0]) * h->dof; }
static int64_t fr_n(const oracle_hmat *h, int64_t k) { return (h->fr[4 * k + 3] - h->fr[4 * k + 1]) * h->dof; }
static int64_t lr_m(const oracle_hmat *h, int64_t k) { return (h->lr[5 * k + 2] - h->lr[5 * k + 0]) * h->dof; }
static int64_t lr_n(const oracle_hmat *h, int64_t k) { return (h->lr[5 * k + 3] - h->lr[5 * k + 1]) * h->dof; }

/* Offsets of each block in the concatenated data arrays. */
static void offsets(const oracle_hmat *h, int64_t *fro, int64_t *lro) {
  int64_t o = 0;
  for (int64_t k = 0; k < h->n_fr; k++) {
    fro[k] = o;
    o += fr_m(h, k) * fr_n(h, k);
  }
  o = 0;
  for (int64_t k = 0; k < h->n_lr; k++) {
    lro[k] = o;
    o += h->lr[5 * k + 4] * (lr_m(h, k) + lr_n(h, k));
  }
}

/* y += A x for a column-major m x n block (il::blas -> cblas_dgemv, beta = 1). */
static void gemv_acc(int64_t m, int64_t n, const double *a, const double *x, double *y) {
  for (int64_t j = 0; j < n; j++) {
    const double xj = x[j];
    const double *col = a + j * m;
    for (int64_t i = 0; i < m; i++) y[i] += col[i] * xj;
  }
}

/* y += A^T x for a column-major m x n block. */
static void gemv_t_acc(int64_t m, int64_t n, const double *a, const double *x, double *y) {
  for (int64_t j = 0; j < n; j++) {
    const double *col = a + j * m;
    double s = 0.0;
    for (int64_t i = 0; i < m; i++) s += col[i] * x[i];
    y[j] += s;
  }
}

/* Hmat<double>::matvec (src/hmat/hmatrix/hmat.cc:472-537): every thread owns a
 * private y; FR blocks do y_i += A x_j (:490-502); LR blocks do t = B x_j then
 * y_i += A t (:509-527); private copies are summed at the end (:532-533).
 * Threads take blocks in a static round-robin and the private copies are
 * summed in thread order, so the result does not depend on timing. */
static int matvec_core(const oracle_hmat *h, const double *x, double *y, int nthreads, int transposed) {
  const int dof = h->dof;
  const int64_t ny = transposed ? h->n_cols : h->n_rows;
  int64_t *fro = (int64_t *)malloc(sizeof(int64_t) * (h->n_fr + 1));
  int64_t *lro = (int64_t *)malloc(sizeof(int64_t) * (h->n_lr + 1));
  if (!fro || !lro) return 1;
  offsets(h, fro, lro);
  if (nthreads < 1) nthreads = 1;
  double *priv = (double *)calloc((size_t)nthreads * (size_t)ny, sizeof(double));
  if (!priv) return 1;
  const int64_t nblk = h->n_fr + h->n_lr;
#pragma omp parallel num_threads(nthreads)
  {
    const int tid = omp_get_thread_num();
    double *yp = priv + (size_t)tid * (size_t)ny;
    double *tmp = NULL;
    int64_t tmp_cap = 0;
    for (int64_t b = tid; b < nblk; b += nthreads) {
      if (b < h->n_fr) {
        const int64_t k = b;
        const int64_t i0 = h->fr[4 * k] * dof, j0 = h->fr[4 * k + 1] * dof;
        const int64_t m = fr_m(h, k), n = fr_n(h, k);
        const double *a = h->fr_data + fro[k];
        if (!transposed)
          gemv_acc(m, n, a, x + j0, yp + i0);
        else
          gemv_t_acc(m, n, a, x + i0, yp + j0);
      } else {
        const int64_t k = b - h->n_fr;
        const int64_t i0 = h->lr[5 * k] * dof, j0 = h->lr[5 * k + 1] * dof;
        const int64_t m = lr_m(h, k), n = lr_n(h, k), r = h->lr[5 * k + 4];
        const double *A = h->lr_data + lro[k];
        const double *B = A + m * r;
        if (r > tmp_cap) {
          free(tmp);
          tmp = (double *)malloc(sizeof(double) * (size_t)r);
          tmp_cap = r;
        }
        memset(tmp, 0, sizeof(double) * (size_t)r);
        if (!transposed) {
          gemv_acc(r, n, B, x + j0, tmp);   /* t = B x_j    (hmat.cc:524) */
          gemv_acc(m, r, A, tmp, yp + i0);  /* y_i += A t   (hmat.cc:526) */
        } else {
          gemv_t_acc(m, r, A, x + i0, tmp); /* s = A^T x_i */
          gemv_t_acc(r, n, B, tmp, yp + j0);/* y_j += B^T s */
        }
      }
    }
    free(tmp);
  }
  for (int64_t i = 0; i < ny; i++) {
    double s = 0.0;
    for (int t = 0; t < nthreads; t++) s += priv[(size_t)t * (size_t)ny + i];
    y[i] = s;
  }
  free(priv);
  free(fro);
  free(lro);
  return 0;
}

int oracle_matvec_perm(const oracle_hmat *h, const double *x, double *y, int nthreads) {
  return matvec_core(h, x, y, nthreads, 0);
}

int oracle_rmatvec_perm(const oracle_hmat *h, const double *x, double *y, int nthreads) {
  return matvec_core(h, x, y, nthreads, 1);
}

/* Hmat<double>::matvecOriginal (hmat.cc:572-635): z[dof*i+j] = x[dof*perm1[i]+j],
 * y = matvec(z), yout[dof*perm0[i]+j] = y[dof*i+j]. */
static int original_core(const oracle_hmat *h, const double *x, double *yout, int nthreads, int transposed) {
  const int dof = h->dof;
  const int64_t nin = transposed ? h->n_rows : h->n_cols;
  const int64_t nout = transposed ? h->n_cols : h->n_rows;
  const int64_t *pin = transposed ? h->perm0 : h->perm1;
  const int64_t *pout = transposed ? h->perm1 : h->perm0;
  double *z = (double *)malloc(sizeof(double) * (size_t)nin);
  double *y = (double *)malloc(sizeof(double) * (size_t)nout);
  if (!z || !y) return 1;
  for (int64_t i = 0; i < nin / dof; i++)
    for (int j = 0; j < dof; j++) z[dof * i + j] = x[dof * pin[i] + j];
  int rc = matvec_core(h, z, y, nthreads, transposed);
  for (int64_t i = 0; i < nout / dof; i++)
    for (int j = 0; j < dof; j++) yout[dof * pout[i] + j] = y[dof * i + j];
  free(z);
  free(y);
  return rc;
}

int oracle_matvec(const oracle_hmat *h, const double *x, double *y, int nthreads) {
  return original_core(h, x, y, nthreads, 0);
}

int oracle_rmatvec(const oracle_hmat *h, const double *x, double *y, int nthreads) {
  return original_core(h, x, y, nthreads, 1);
}

int oracle_matmat(const oracle_hmat *h, const double *X, double *Y, int64_t k, int nthreads) {
  for (int64_t c = 0; c < k; c++) {
    int rc = original_core(h, X + c * h->n_cols, Y + c * h->n_rows, nthreads, 0);
    if (rc) return rc;
  }
  return 0;
}

/* Hmat::diagonal (hmat.cc:256-285) then the permutation back of
 * Hmat::diagonalOriginal (hmat.cc:240-254).  A FR block contributes the
 * entries (i, j) with i + dof*i0 == j + dof*j0; blocks that lie strictly
 * below or above the diagonal are skipped exactly as the reference tests them. */
int oracle_diagonal(const oracle_hmat *h, double *d) {
  const int dof = h->dof;
  const int64_t n = h->n_rows > h->n_cols ? h->n_rows : h->n_cols;
  double *raw = (double *)calloc((size_t)n, sizeof(double));
  int64_t *fro = (int64_t *)malloc(sizeof(int64_t) * (h->n_fr + 1));
  int64_t *lro = (int64_t *)malloc(sizeof(int64_t) * (h->n_lr + 1));
  if (!raw || !fro || !lro) return 1;
  offsets(h, fro, lro);
  for (int64_t k = 0; k < h->n_fr; k++) {
    const int64_t i0 = h->fr[4 * k], j0 = h->fr[4 * k + 1], iend = h->fr[4 * k + 2], jend = h->fr[4 * k + 3];
    const int in_lower = (i0 > j0) && (i0 > jend) && (iend > j0) && (iend > jend);
    const int in_upper = (i0 < j0) && (i0 < jend) && (iend < j0) && (iend < jend);
    if (in_lower || in_upper) continue;
    const int64_t m = fr_m(h, k), nn = fr_n(h, k);
    const double *a = h->fr_data + fro[k];
    for (int64_t j = 0; j < nn; j++)
      for (int64_t i = 0; i < m; i++)
        if (i + dof * i0 == j + dof * j0) raw[i + dof * i0] = a[i + j * m];
  }
  memset(d, 0, sizeof(double) * (size_t)n);
  for (int64_t i = 0; i < n / dof; i++)
    for (int j = 0; j < dof; j++) d[dof * h->perm1[i] + j] = raw[dof * i + j];
  free(raw);
  free(fro);
  free(lro);
  return 0;
}

int64_t oracle_entries(const oracle_hmat *h) {
  int64_t s = 0;
  for (int64_t k = 0; k < h->n_fr; k++) s += fr_m(h, k) * fr_n(h, k);
  for (int64_t k = 0; k < h->n_lr; k++) s += h->lr[5 * k + 4] * (lr_m(h, k) + lr_n(h, k));
  return s;
}
