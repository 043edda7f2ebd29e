// Laying out device-resident blocks on the device (bw_add_flat_device):
// the three data passes of bw_finalize that otherwise run on the host.
//   * block_maxabs_kernel: max |entry| and a non-finite flag per stored block
//     (full-rank block, low-rank A, low-rank B): the inputs of
//     scales_from_maxima, which gives compute_scales' scales bit for bit;
//   * pack_runs_kernel<PREC>: the layout fill as PackRuns (build_pack_runs),
//     each element through bw::pack::element, which equals the host fill
//     byte for byte;
//   * diag_kernel: the diagonal entries of the full-rank blocks that cross the
//     diagonal (Hmat::diagonal, src/hmat/hmatrix/hmat.cc:256-285).
// One CTA per span / run / block (grid-stride); every offset was checked on
// the host against the array lengths before the launch.
#pragma once

#include "bw_pack.h"

namespace bw {

constexpr int kDevLayoutThreads = 256;

struct MaxSpan {
  long long off;         // first element in its array
  long long rows, cols;  // column-major, leading dimension rows
  int array, pad;        // 0: full-rank data, 1: low-rank data
};

struct DiagSpan {
  long long off;       // block's first element in the full-rank data
  long long m;         // rows (leading dimension)
  long long i0, j0;    // block position (scalar rows / columns)
  long long lo, hi;    // diagonal indices d in [lo, hi) the block holds
};

__global__ void __launch_bounds__(kDevLayoutThreads) block_maxabs_kernel(const MaxSpan *__restrict__ spans, int n,
                                                                         const double *__restrict__ fr,
                                                                         const double *__restrict__ lr,
                                                                         double *__restrict__ out_max,
                                                                         int *__restrict__ out_bad) {
  __shared__ double s_max[kDevLayoutThreads];
  __shared__ int s_bad[kDevLayoutThreads];
  const int t = threadIdx.x;
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const MaxSpan sp = spans[k];
    const double *base = (sp.array == 0 ? fr : lr) + sp.off;
    const long long total = sp.rows * sp.cols;
    double m = 0.0;
    int bad = 0;
    for (long long e = t; e < total; e += kDevLayoutThreads) {
      const double a = fabs(base[e]);
      if (!(a <= 1.0e300)) bad = 1;
      m = fmax(m, a);  // NaN never wins (the host max of |entries| keeps the larger operand too)
    }
    s_max[t] = m;
    s_bad[t] = bad;
    __syncthreads();
    for (int s = kDevLayoutThreads / 2; s > 0; s >>= 1) {
      if (t < s) {
        s_max[t] = fmax(s_max[t], s_max[t + s]);
        s_bad[t] |= s_bad[t + s];
      }
      __syncthreads();
    }
    if (t == 0) {
      out_max[k] = s_max[0];
      out_bad[k] = s_bad[0];
    }
    __syncthreads();
  }
}

template <int PREC>
__global__ void __launch_bounds__(kDevLayoutThreads) pack_runs_kernel(const PackRun *__restrict__ runs,
                                                                      long long n_runs,
                                                                      const double *__restrict__ fr,
                                                                      const double *__restrict__ lr, void *dst) {
  for (long long k = blockIdx.x; k < n_runs; k += gridDim.x) {
    const PackRun r = runs[k];
    const long long total = (long long)r.n * r.ncols;
    for (long long e = threadIdx.x; e < total; e += kDevLayoutThreads) {
      const long long c = e / r.n, i = e - c * r.n;  // consecutive threads: consecutive rows of one column
      pack::element<PREC>(dst, r, fr, lr, i, c);
    }
  }
}

__global__ void __launch_bounds__(kDevLayoutThreads) diag_kernel(const DiagSpan *__restrict__ spans, int n,
                                                                 const double *__restrict__ fr,
                                                                 double *__restrict__ diag) {
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const DiagSpan sp = spans[k];
    for (long long d = sp.lo + threadIdx.x; d < sp.hi; d += kDevLayoutThreads)
      diag[d] = fr[sp.off + (d - sp.i0) + (d - sp.j0) * sp.m];
  }
}

}  // namespace bw
