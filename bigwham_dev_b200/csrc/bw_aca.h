// Block adaptive cross approximation of one admissible block, for host and
// device code.
//
// The reference compresses every admissible block with a block-pivoted ACA
// (adaptiveCrossApproximation<p>, src/hmat/compression/
// adaptiveCrossApproximation.h:24-226, routines in routines.h:46-188), with
// p x p pivot blocks, p = dof.  This header restates that algorithm:
//   step k, with row block i0 (initially the first):
//   * residual row band R = M(i0, :) - A(i0, :) B (p x n1 p);
//   * pivot column block i1: among column blocks not used yet, the one whose
//     p x p block of R has the largest SMALLEST singular value (the first one
//     on ties); none left (all zero) -> stop;
//   * Gamma = inverse of that p x p block (stop if not finite);
//   * A_k = residual column band M(:, i1) - A B(:, i1) (n0 p x p);
//     B_k = Gamma R (recomputed residual row, p x n1 p);
//   * |A_k B_k|_F^2 and 2 sum_{r<k} <A_r B_r, A_k B_k>_F update the squared
//     Frobenius norm S of the approximation;
//   * next row block: among row blocks not used yet, the one whose p x p
//     block of A_k has the largest smallest singular value;
//   * stop when no row block is left, when the rank reaches min(n0, n1)
//     blocks, or when |A_k B_k|_F^2 <= eps^2 S; the error estimate is
//     sqrt(|A_k B_k|_F^2 / S) (LowRank::error_on_approximation).
// The result is A (n0 p x r p) and B (r p x n1 p), column-major, rank r p.
// Singular values here come from Jacobi rotations on the 3 x 3 Gram matrix
// and inverses from Gauss-Jordan elimination with partial pivoting; the
// reference uses LAPACK for both, so pivots can differ where candidate
// singular values tie to rounding, and with them the factors; the accuracy
// bound is the same.
#pragma once

#include <cmath>

#include "bw_r0.h"

namespace bw {
namespace aca {

// The pivot blocks are P x P, P = dof: 3 for the 3D elastic kernels, 2 for
// the 2D ones.  The P = 3 entry points below (smallest_singular_value,
// invert3) are the ones the device kernel calls.

// Smallest singular value of a P x P matrix m (column-major): square root of
// the smallest eigenvalue of m^T m by cyclic Jacobi rotations.
template <int P>
BW_HD double smallest_singular_value_p(const double *m) {
  double g[P][P];
  for (int a = 0; a < P; a++)
    for (int b = 0; b < P; b++) {
      double s = 0.0;
      for (int k = 0; k < P; k++) s += m[a * P + k] * m[b * P + k];
      g[a][b] = s;
    }
  for (int sweep = 0; sweep < 12; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int p = 0; p < P; p++)
      for (int q = p + 1; q < P; q++) off += g[p][q] * g[p][q];
    for (int p = 0; p < P; p++) diag += g[p][p] * g[p][p];
    if (off <= 1e-36 * diag) break;
    for (int p = 0; p < P - 1; p++)
      for (int q = p + 1; q < P; q++) {
        if (g[p][q] == 0.0) continue;
        const double theta = (g[q][q] - g[p][p]) / (2.0 * g[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < P; k++) {  // columns p, q
          const double gkp = g[k][p], gkq = g[k][q];
          g[k][p] = c * gkp - s * gkq;
          g[k][q] = s * gkp + c * gkq;
        }
        for (int k = 0; k < P; k++) {  // rows p, q
          const double gpk = g[p][k], gqk = g[q][k];
          g[p][k] = c * gpk - s * gqk;
          g[q][k] = s * gpk + c * gqk;
        }
      }
  }
  double lmin = g[P - 1][P - 1];
  for (int p = P - 2; p >= 0; p--) lmin = fmin(g[p][p], lmin);
  return lmin > 0.0 ? sqrt(lmin) : 0.0;
}

BW_HD double smallest_singular_value(const double *m) { return smallest_singular_value_p<3>(m); }

// Inverse of a P x P matrix (column-major) by Gauss-Jordan elimination with
// partial pivoting; false if a pivot is zero or the inverse is not finite.
template <int P>
BW_HD bool invert_p(const double *m, double *inv) {
  double a[P][2 * P];
  for (int r = 0; r < P; r++)
    for (int c = 0; c < P; c++) {
      a[r][c] = m[c * P + r];
      a[r][P + c] = r == c ? 1.0 : 0.0;
    }
  for (int c = 0; c < P; c++) {
    int piv = c;
    for (int r = c + 1; r < P; r++)
      if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
    if (a[piv][c] == 0.0) return false;
    if (piv != c)
      for (int k = 0; k < 2 * P; k++) {
        const double t = a[c][k];
        a[c][k] = a[piv][k];
        a[piv][k] = t;
      }
    const double d = 1.0 / a[c][c];
    for (int k = 0; k < 2 * P; k++) a[c][k] *= d;
    for (int r = 0; r < P; r++)
      if (r != c) {
        const double f = a[r][c];
        if (f != 0.0)
          for (int k = 0; k < 2 * P; k++) a[r][k] -= f * a[c][k];
      }
  }
  for (int r = 0; r < P; r++)
    for (int c = 0; c < P; c++) inv[c * P + r] = a[r][P + c];
  for (int k = 0; k < P * P; k++)
    if (!(fabs(inv[k]) <= 1.7976931348623157e308)) return false;  // NaN or infinite
  return true;
}

BW_HD bool invert3(const double *m, double *inv) { return invert_p<3>(m, inv); }

struct Result {
  int rank_blocks;  // rank / P
  double error;     // error estimate (0 when the loop stopped otherwise)
  bool overflow;    // stopped because the factor storage was full
};

// Host (sequential) block ACA.  entry(i, j, K) writes the P x P block of
// point row i (0 <= i < n0) and point column j (0 <= j < n1), K[a][b] =
// row a, column b.  A: n0 P x cap P, B: cap P x n1 P column-major buffers;
// work: (n0 + n1) P x P + n0 + n1 doubles.  Stops at cap blocks of rank.
template <int P = 3, typename Entry>
Result block_aca_host(const Entry &entry, int n0, int n1, double eps, int cap, double *A, double *B, double *work) {
  const long long lda = (long long)n0 * P, ldb = (long long)cap * P;
  double *row = work;                               // P x n1 P, column-major (ld P)
  double *col = row + (long long)P * n1 * P;        // n0 P x P, column-major (ld n0 P)
  double *used0 = col + (long long)n0 * P * P;      // n0 flags
  double *used1 = used0 + n0;                       // n1 flags
  for (int i = 0; i < n0; i++) used0[i] = 0.0;
  for (int j = 0; j < n1; j++) used1[j] = 0.0;
  Result res = {0, 0.0, false};
  int i0 = 0, rank = 0;
  double s_norm = 0.0;
  const int max_rank = n0 < n1 ? n0 : n1;
  auto residual_row = [&](int ip) {
    for (int j = 0; j < n1; j++) {
      double K[P][P];
      entry(ip, j, K);
      for (int b = 0; b < P; b++)
        for (int a = 0; a < P; a++) {
          double v = K[a][b];
          for (int k = 0; k < rank * P; k++) v -= A[k * lda + ip * P + a] * B[(long long)(j * P + b) * ldb + k];
          row[(long long)(j * P + b) * P + a] = v;
        }
    }
  };
  while (true) {
    if (rank >= cap) {
      res.overflow = true;
      break;
    }
    residual_row(i0);
    int i1 = -1;
    double best = 0.0;
    for (int j = 0; j < n1; j++) {
      if (used1[j] != 0.0) continue;
      const double sv = smallest_singular_value_p<P>(row + (long long)j * P * P);
      if (sv > best) {
        best = sv;
        i1 = j;
      }
    }
    if (i1 < 0) break;
    used0[i0] = 1.0;
    used1[i1] = 1.0;
    double gamma[P * P];
    if (!invert_p<P>(row + (long long)i1 * P * P, gamma)) break;
    // A_k: residual column band
    for (int i = 0; i < n0; i++) {
      double K[P][P];
      entry(i, i1, K);
      for (int b = 0; b < P; b++)
        for (int a = 0; a < P; a++) {
          double v = K[a][b];
          for (int k = 0; k < rank * P; k++) v -= A[k * lda + i * P + a] * B[(long long)(i1 * P + b) * ldb + k];
          col[(long long)b * lda + i * P + a] = v;
        }
    }
    for (int b = 0; b < P; b++)
      for (long long r = 0; r < lda; r++) A[(long long)(rank * P + b) * lda + r] = col[(long long)b * lda + r];
    // B_k = Gamma R (the residual row again, as the reference recomputes it)
    residual_row(i0);
    for (int j = 0; j < n1 * P; j++)
      for (int a = 0; a < P; a++) {
        double v = 0.0;
        for (int c = 0; c < P; c++) v += gamma[c * P + a] * row[(long long)j * P + c];
        B[(long long)j * ldb + rank * P + a] = v;
      }
    // |A_k B_k|_F^2 = sum (A_k^T A_k) .* (B_k B_k^T)
    double ata[P * P] = {}, bbt[P * P] = {};
    for (int a = 0; a < P; a++)
      for (int b = 0; b < P; b++) {
        double sa = 0.0, sb = 0.0;
        for (long long r = 0; r < lda; r++) sa += A[(long long)(rank * P + a) * lda + r] * A[(long long)(rank * P + b) * lda + r];
        for (int j = 0; j < n1 * P; j++) sb += B[(long long)j * ldb + rank * P + a] * B[(long long)j * ldb + rank * P + b];
        ata[b * P + a] = sa;
        bbt[b * P + a] = sb;
      }
    double ab = 0.0;
    for (int k = 0; k < P * P; k++) ab += ata[k] * bbt[k];
    // cross terms 2 sum_r <A_r B_r, A_k B_k> = 2 sum_r trace((A_r^T A_k)(B_k B_r^T))
    double cross = 0.0;
    for (int r = 0; r < rank; r++) {
      double m1[P * P], m2[P * P];
      for (int a = 0; a < P; a++)
        for (int b = 0; b < P; b++) {
          double s1 = 0.0, s2 = 0.0;
          for (long long q = 0; q < lda; q++) s1 += A[(long long)(r * P + a) * lda + q] * A[(long long)(rank * P + b) * lda + q];
          for (int j = 0; j < n1 * P; j++) s2 += B[(long long)j * ldb + rank * P + b] * B[(long long)j * ldb + r * P + a];
          m1[b * P + a] = s1;  // (A_r^T A_k)(a, b)
          m2[b * P + a] = s2;  // (B_k B_r^T)(b, a) stored at (a, b)
        }
      for (int k = 0; k < P * P; k++) cross += m1[k] * m2[k];
    }
    s_norm += 2.0 * cross + ab;
    // next row block from A_k
    int next = -1;
    best = 0.0;
    for (int i = 0; i < n0; i++) {
      if (used0[i] != 0.0) continue;
      double blk[P * P];
      for (int b = 0; b < P; b++)
        for (int a = 0; a < P; a++) blk[b * P + a] = A[(long long)(rank * P + b) * lda + i * P + a];
      const double sv = smallest_singular_value_p<P>(blk);
      if (sv > best) {
        best = sv;
        next = i;
      }
    }
    rank++;
    res.rank_blocks = rank;
    if (next < 0 || rank == max_rank) break;
    if (fabs(ab) <= eps * eps * fabs(s_norm)) {
      res.error = sqrt(fabs(ab) / fabs(s_norm));
      break;
    }
    i0 = next;
  }
  res.rank_blocks = rank;
  return res;
}

}  // namespace aca
}  // namespace bw
