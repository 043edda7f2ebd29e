// Device block ACA of the admissible blocks of a 3DR0-H H-matrix.
//
// One CTA compresses one block at a time (grid-stride over blocks), running
// the steps of bw::aca::block_aca_host with the work of each step spread over
// the CTA's threads:
//   * residual row / column bands: one thread per point pair (kernel entry +
//     the subtraction of the current approximation);
//   * pivot searches: per-thread smallest singular values, then a CTA argmax
//     that keeps the first index on ties (the reference scans in order and
//     replaces only on a strictly larger value);
//   * Frobenius terms: CTA reductions of 3 x 3 Gram blocks.
// Every stop decision is taken by thread 0 and broadcast through shared
// memory, so all threads leave the loop together.  Factor storage per block is
// capacity-bounded (cap blocks of rank); a block that needs more reports
// rank -1 and writes nothing past its capacity.
#pragma once

#include "bw_aca.h"
#include "bw_r0.h"

namespace bw {

constexpr int kAcaThreads = 128;

struct AcaBlock {
  long long a_off, b_off;  // factor storage (doubles): A n0 3 x cap 3, B cap 3 x n1 3, column-major
  long long s_off;         // unused here (kept for alignment of the record)
  int i0, j0, n0, n1;      // first row / column point (permuted numbering), sizes in points
  int cap, pad;            // rank capacity in blocks
};

// CTA argmax of (value, index) pairs: largest value, smallest index on ties;
// index -1 when no thread had a candidate.
__device__ __forceinline__ void aca_argmax(double v, int idx, double *sv, int *si, double &best, int &bi) {
  const int t = threadIdx.x;
  sv[t] = v;
  si[t] = idx;
  __syncthreads();
  for (int s = kAcaThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      const double v2 = sv[t + s];
      const int i2 = si[t + s];
      if (i2 >= 0 && (si[t] < 0 || v2 > sv[t] || (v2 == sv[t] && i2 < si[t]))) {
        sv[t] = v2;
        si[t] = i2;
      }
    }
    __syncthreads();
  }
  best = sv[0];
  bi = si[0];
  __syncthreads();
}

// CTA sum of 9 partial values per thread into out[9] (all threads see it).
__device__ __forceinline__ void aca_sum9(const double *part, double *red, double *out) {
  const int t = threadIdx.x;
  for (int k = 0; k < 9; k++) red[k * kAcaThreads + t] = part[k];
  __syncthreads();
  for (int s = kAcaThreads / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int k = 0; k < 9; k++) red[k * kAcaThreads + t] += red[k * kAcaThreads + t + s];
    __syncthreads();
  }
  for (int k = 0; k < 9; k++) out[k] = red[k * kAcaThreads];
  __syncthreads();
}

__global__ void __launch_bounds__(kAcaThreads) r0_aca_kernel(const double *__restrict__ records,
                                                             const int *__restrict__ perm,
                                                             const AcaBlock *__restrict__ blocks, int n_blocks,
                                                             double G, double nu, double eps, double *factors_a,
                                                             double *factors_b, double *scratch,
                                                             long long slot_doubles, int *rank_out,
                                                             double *err_out) {
  __shared__ double s_val[kAcaThreads];
  __shared__ int s_idx[kAcaThreads];
  __shared__ double s_red[9 * kAcaThreads];
  __shared__ double s_gamma[9];
  __shared__ int s_ctl[4];  // [0] continue, [1] next row block, [2] pivot column block
  const int t = threadIdx.x;
  double *row = scratch + (long long)blockIdx.x * slot_doubles;  // 3 x n1 3 (ld 3)
  for (int bk = blockIdx.x; bk < n_blocks; bk += gridDim.x) {
    const AcaBlock B_ = blocks[bk];
    const int n0 = B_.n0, n1 = B_.n1, cap = B_.cap;
    const long long lda = 3LL * n0, ldb = 3LL * cap;
    double *A = factors_a + B_.a_off;
    double *Bf = factors_b + B_.b_off;
    int *used0 = reinterpret_cast<int *>(row + 9LL * n1);
    int *used1 = used0 + n0;
    for (int i = t; i < n0; i += kAcaThreads) used0[i] = 0;
    for (int j = t; j < n1; j += kAcaThreads) used1[j] = 0;
    __syncthreads();
    auto entry = [&](int i, int j, double K[3][3]) {
      const double *src = records + r0::kFrameDoubles * perm[B_.j0 + j];
      const double *rec = records + r0::kFrameDoubles * perm[B_.i0 + i];
      r0::influence_h(src, src + 3, src[15], src[16], rec, rec + 3, rec + 12, G, nu, K);
    };
    int rank = 0, i0 = 0, status = 0;  // status: 0 running, 1 done, 2 overflow
    double s_norm = 0.0, err = 0.0;
    const int max_rank = n0 < n1 ? n0 : n1;
    while (status == 0) {
      if (rank >= cap) {
        status = 2;
        break;
      }
      // residual row band of row block i0
      for (int j = t; j < n1; j += kAcaThreads) {
        double K[3][3];
        entry(i0, j, K);
        for (int b = 0; b < 3; b++)
          for (int a = 0; a < 3; a++) {
            double v = K[a][b];
            for (int k = 0; k < 3 * rank; k++) v -= A[k * lda + 3LL * i0 + a] * Bf[(3LL * j + b) * ldb + k];
            row[(3LL * j + b) * 3 + a] = v;
          }
      }
      __syncthreads();
      // pivot column block
      double best = 0.0;
      int bi = -1;
      for (int j = t; j < n1; j += kAcaThreads) {
        if (used1[j]) continue;
        const double sv = aca::smallest_singular_value(row + 9LL * j);
        if (sv > best) {  // ascending j per thread: the first maximum stays
          best = sv;
          bi = j;
        }
      }
      double gbest;
      int i1;
      aca_argmax(best, bi, s_val, s_idx, gbest, i1);
      if (i1 < 0) break;  // uniform: every thread read the same i1
      if (t == 0) {
        used0[i0] = 1;
        used1[i1] = 1;
        s_ctl[0] = aca::invert3(row + 9LL * i1, s_gamma) ? 1 : 0;
      }
      __syncthreads();
      if (!s_ctl[0]) break;
      // A_k: residual column band of column block i1
      for (int i = t; i < n0; i += kAcaThreads) {
        double K[3][3];
        entry(i, i1, K);
        for (int b = 0; b < 3; b++)
          for (int a = 0; a < 3; a++) {
            double v = K[a][b];
            for (int k = 0; k < 3 * rank; k++) v -= A[k * lda + 3LL * i + a] * Bf[(3LL * i1 + b) * ldb + k];
            A[(3LL * rank + b) * lda + 3LL * i + a] = v;
          }
      }
      // B_k = Gamma R
      for (int j = t; j < 3 * n1; j += kAcaThreads)
        for (int a = 0; a < 3; a++) {
          double v = 0.0;
          for (int c = 0; c < 3; c++) v += s_gamma[c * 3 + a] * row[3LL * j + c];
          Bf[(long long)j * ldb + 3LL * rank + a] = v;
        }
      __syncthreads();
      // |A_k B_k|_F^2 and cross terms with the earlier rank blocks
      double part[9], ata[9], bbt[9];
      for (int k = 0; k < 9; k++) part[k] = 0.0;
      for (long long r = t; r < lda; r += kAcaThreads)
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            part[b * 3 + a] += A[(3LL * rank + a) * lda + r] * A[(3LL * rank + b) * lda + r];
      aca_sum9(part, s_red, ata);
      for (int k = 0; k < 9; k++) part[k] = 0.0;
      for (long long j = t; j < 3LL * n1; j += kAcaThreads)
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) part[b * 3 + a] += Bf[j * ldb + 3LL * rank + a] * Bf[j * ldb + 3LL * rank + b];
      aca_sum9(part, s_red, bbt);
      double ab = 0.0;
      for (int k = 0; k < 9; k++) ab += ata[k] * bbt[k];
      double cross = 0.0;
      for (int r = 0; r < rank; r++) {
        double m1[9], m2[9];
        for (int k = 0; k < 9; k++) part[k] = 0.0;
        for (long long q = t; q < lda; q += kAcaThreads)
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) part[b * 3 + a] += A[(3LL * r + a) * lda + q] * A[(3LL * rank + b) * lda + q];
        aca_sum9(part, s_red, m1);
        for (int k = 0; k < 9; k++) part[k] = 0.0;
        for (long long j = t; j < 3LL * n1; j += kAcaThreads)
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) part[b * 3 + a] += Bf[j * ldb + 3LL * rank + b] * Bf[j * ldb + 3LL * r + a];
        aca_sum9(part, s_red, m2);
        for (int k = 0; k < 9; k++) cross += m1[k] * m2[k];
      }
      s_norm += 2.0 * cross + ab;
      // next row block from A_k
      best = 0.0;
      bi = -1;
      for (int i = t; i < n0; i += kAcaThreads) {
        if (used0[i]) continue;
        double blk[9];
        for (int b = 0; b < 3; b++)
          for (int a = 0; a < 3; a++) blk[b * 3 + a] = A[(3LL * rank + b) * lda + 3LL * i + a];
        const double sv = aca::smallest_singular_value(blk);
        if (sv > best) {
          best = sv;
          bi = i;
        }
      }
      int next;
      aca_argmax(best, bi, s_val, s_idx, gbest, next);
      rank++;
      if (next < 0 || rank == max_rank) break;
      if (fabs(ab) <= eps * eps * fabs(s_norm)) {
        err = sqrt(fabs(ab) / fabs(s_norm));
        break;
      }
      i0 = next;
    }
    if (t == 0) {
      rank_out[bk] = status == 2 ? -1 : rank;
      err_out[bk] = err;
    }
    __syncthreads();
  }
}

}  // namespace bw
