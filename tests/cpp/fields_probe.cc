// Host builds of the observation-field code the device kernels run per
// (point, element) pair, in the kernels' order (per point, elements in mesh
// order): 2DS0 (bigwham_dev_b200/csrc/bw_s0.h, s0_fields_kernel) and 3DR0
// (bw_r0_fields.h, r0_fields_kernel).  Test helper: compiled by
// tests/test_fields_cpu.py with g++.
#include "bw_aca.h"
#include "bw_r0_fields.h"
#include "bw_s0.h"

#include <cstdint>

extern "C" int probe_s0_fields(int64_t n_elems, const double *rec, const double *dd, double G, double nu,
                               int64_t n_pts, const double *pts, double *stress, double *disp) {
  for (int64_t p = 0; p < n_pts; p++) {
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t e = 0; e < n_elems; e++)
      bw::s0::add_point_fields(rec + bw::s0::kRecordDoubles * e, dd[2 * e], dd[2 * e + 1], pts[2 * p],
                               pts[2 * p + 1], G, nu, acc);
    for (int k = 0; k < 3; k++) stress[3 * p + k] = acc[k];
    for (int k = 0; k < 2; k++) disp[2 * p + k] = acc[3 + k];
  }
  return 0;
}

// records: n_elems x 17 (the assembly records); the element values are packed
// as r0_fields_kernel stages them.
extern "C" int probe_r0_fields(int64_t n_elems, const double *rec, const double *dd, double G, double nu,
                               int64_t n_pts, const double *pts, double *stress, double *disp) {
  for (int64_t p = 0; p < n_pts; p++) {
    double acc[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t e = 0; e < n_elems; e++) {
      double el[bw::r0::kFieldDoubles];
      for (int k = 0; k < 14; k++) el[k] = rec[bw::r0::kFrameDoubles * e + (k < 12 ? k : k + 3)];
      for (int k = 0; k < 3; k++) el[14 + k] = dd[3 * e + k];
      bw::r0::add_point_fields(el, pts + 3 * p, G, nu, acc);
    }
    for (int k = 0; k < 6; k++) stress[6 * p + k] = acc[k];
    for (int k = 0; k < 3; k++) disp[3 * p + k] = acc[6 + k];
  }
  return 0;
}

// Dense 2DS0 H matrix (original element order, 2 x 2 per pair) from
// bw::s0::h_entry: H[(2 i + j), (2 e + k)] = traction j at element i due to
// DD k of element e; out is (2 n) x (2 n) row-major.
extern "C" int probe_s0_dense_h(int64_t n, const double *rec, double G, double nu, double *out) {
  for (int64_t i = 0; i < n; i++)
    for (int64_t e = 0; e < n; e++) {
      double K[2][2];
      bw::s0::h_entry(rec + 5 * e, rec + 5 * i, G, nu, K);
      for (int j = 0; j < 2; j++)
        for (int k = 0; k < 2; k++) out[(2 * i + j) * 2 * n + 2 * e + k] = K[j][k];
    }
  return 0;
}

// Block ACA with 2 x 2 pivots (bw::aca::block_aca_host<2>) of the 2DS0 block
// [i0, i1) x [j0, j1) (permuted points; perm: permuted point -> element) with
// the entries of bw::s0::h_entry.  A: (i1 - i0) 2 x cap 2, B: cap 2 x
// (j1 - j0) 2, column-major; returns the rank in blocks (-1 when cap was too
// small).
extern "C" int probe_s0_aca(const double *rec, double G, double nu, const int64_t *perm, int64_t i0, int64_t j0,
                            int64_t i1, int64_t j1, double eps, int cap, double *A, double *B, double *err) {
  const int n0 = (int)(i1 - i0), n1 = (int)(j1 - j0);
  double *work = new double[(size_t)(n0 + n1) * 4 + n0 + n1];
  auto entry = [&](int i, int j, double K[2][2]) {
    bw::s0::h_entry(rec + 5 * perm[j0 + j], rec + 5 * perm[i0 + i], G, nu, K);
  };
  const bw::aca::Result r = bw::aca::block_aca_host<2>(entry, n0, n1, eps, cap, A, B, work);
  delete[] work;
  *err = r.error;
  return r.overflow ? -1 : r.rank_blocks;
}
