// Host build of the 2DS0 observation-field code (bigwham_dev_b200/csrc/bw_s0.h),
// the same functions s0_fields_kernel runs per (point, element) pair, in the
// kernel's order (per point, elements in mesh order).  Test helper: compiled
// by tests/test_fields_cpu.py with g++.
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

// Local fields of unit DDs at (x, y) for a segment of half length a:
// s (2 x 3: per DD shear / normal, sxx syy sxy), u (2 x 2: ux uy).
extern "C" int probe_s0_local(double x, double y, double a, double G, double nu, double *s, double *u) {
  double ss[2][3], uu[2][2];
  bw::s0::local_fields(x, y, a, G, nu, ss, uu);
  for (int k = 0; k < 2; k++) {
    for (int j = 0; j < 3; j++) s[3 * k + j] = ss[k][j];
    for (int j = 0; j < 2; j++) u[2 * k + j] = uu[k][j];
  }
  return 0;
}
