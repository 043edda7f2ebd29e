// Stresses and displacements at observation points from a 2DS0 solution
// (the reference's BigWhamIO::ComputeStresses / ComputeDisplacements,
// src/io/bigwham_io.cc:1166-1324, on segment meshes): for every point the sum
// over all elements of the element's field times its local DD (bw_s0.h).
//
// One thread per observation point; the CTA stages tiles of element records
// and DDs in shared memory, which all its threads read in the same order
// (broadcast reads).  Each point sums the elements in mesh order, the order
// of the reference's loop.  Per (point, element) pair the work is two
// logarithms, two atan2 and a dozen FP64 divisions: the kernel is bound by
// FP64 arithmetic, not memory (7 doubles per element per tile, reused by 256
// points).
#pragma once

#include "bw_r0_fields.h"
#include "bw_s0.h"

namespace bw {

constexpr int kS0Threads = 256;  // observation points per CTA pass
constexpr int kS0Tile = 256;     // elements per shared-memory tile
constexpr int kS0TileDoubles = 7;

__global__ void __launch_bounds__(kS0Threads) s0_fields_kernel(const double *__restrict__ rec,
                                                               const double *__restrict__ dd, int n_elems,
                                                               const double *__restrict__ pts, long long n_pts,
                                                               double G, double nu, double *__restrict__ stress,
                                                               double *__restrict__ disp) {
  __shared__ double s_el[kS0Tile * kS0TileDoubles];  // per element: cx, cy, a, tx, ty, dd_s, dd_n
  for (long long p0 = static_cast<long long>(blockIdx.x) * kS0Threads; p0 < n_pts;
       p0 += static_cast<long long>(gridDim.x) * kS0Threads) {  // uniform over the CTA
    const long long p = p0 + threadIdx.x;
    const bool live = p < n_pts;
    const double px = live ? pts[2 * p] : 0.0, py = live ? pts[2 * p + 1] : 0.0;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int e0 = 0; e0 < n_elems; e0 += kS0Tile) {
      const int ne = min(kS0Tile, n_elems - e0);
      __syncthreads();  // the previous tile is no longer read
      for (int q = threadIdx.x; q < ne * s0::kRecordDoubles; q += kS0Threads)
        s_el[(q / s0::kRecordDoubles) * kS0TileDoubles + q % s0::kRecordDoubles] =
            rec[static_cast<long long>(e0) * s0::kRecordDoubles + q];
      for (int q = threadIdx.x; q < ne * 2; q += kS0Threads)
        s_el[(q / 2) * kS0TileDoubles + s0::kRecordDoubles + (q & 1)] = dd[2 * static_cast<long long>(e0) + q];
      __syncthreads();
      if (live) {
        for (int e = 0; e < ne; e++) {
          const double *r = s_el + e * kS0TileDoubles;
          s0::add_point_fields(r, r[5], r[6], px, py, G, nu, acc);
        }
      }
    }
    if (live) {
      if (stress) {
        stress[3 * p] = acc[0];
        stress[3 * p + 1] = acc[1];
        stress[3 * p + 2] = acc[2];
      }
      if (disp) {
        disp[2 * p] = acc[3];
        disp[2 * p + 1] = acc[4];
      }
    }
  }
}

constexpr int kR0FieldThreads = 128;  // observation points per CTA pass
constexpr int kR0FieldTile = 128;     // elements per shared-memory tile

// 3DR0: as s0_fields_kernel, with the element's kFieldDoubles values (taken
// from the 17-double assembly records and the local DDs) staged per tile.
__global__ void __launch_bounds__(kR0FieldThreads) r0_fields_kernel(const double *__restrict__ rec,
                                                                    const double *__restrict__ dd, int n_elems,
                                                                    const double *__restrict__ pts, long long n_pts,
                                                                    double G, double nu, double *__restrict__ stress,
                                                                    double *__restrict__ disp) {
  __shared__ double s_el[kR0FieldTile * r0::kFieldDoubles];
  for (long long p0 = static_cast<long long>(blockIdx.x) * kR0FieldThreads; p0 < n_pts;
       p0 += static_cast<long long>(gridDim.x) * kR0FieldThreads) {  // uniform over the CTA
    const long long p = p0 + threadIdx.x;
    const bool live = p < n_pts;
    double q[3] = {0.0, 0.0, 0.0};
    if (live)
      for (int k = 0; k < 3; k++) q[k] = pts[3 * p + k];
    double acc[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int e0 = 0; e0 < n_elems; e0 += kR0FieldTile) {
      const int ne = min(kR0FieldTile, n_elems - e0);
      __syncthreads();  // the previous tile is no longer read
      // record layout: cp 0-2, rotation 3-11, normal 12-14, a 15, b 16
      for (int w = threadIdx.x; w < ne * 14; w += kR0FieldThreads) {
        const int e = w / 14, k = w % 14;
        s_el[e * r0::kFieldDoubles + k] =
            rec[static_cast<long long>(e0 + e) * r0::kFrameDoubles + (k < 12 ? k : k + 3)];
      }
      for (int w = threadIdx.x; w < ne * 3; w += kR0FieldThreads)
        s_el[(w / 3) * r0::kFieldDoubles + 14 + w % 3] = dd[3 * static_cast<long long>(e0) + w];
      __syncthreads();
      if (live)
        for (int e = 0; e < ne; e++) r0::add_point_fields(s_el + e * r0::kFieldDoubles, q, G, nu, acc);
    }
    if (live) {
      if (stress)
        for (int k = 0; k < 6; k++) stress[6 * p + k] = acc[k];
      if (disp)
        for (int k = 0; k < 3; k++) disp[3 * p + k] = acc[6 + k];
    }
  }
}

}  // namespace bw
