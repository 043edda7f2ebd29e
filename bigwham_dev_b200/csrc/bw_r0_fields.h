// Fields at a point due to a rectangular element carrying a constant
// displacement discontinuity (3DR0), in the global frame, host and device:
// the element's local stresses and displacements (bw_r0.h: the reference's
// StressesKernelR0 / DisplacementKernelR0 restated) contracted with the local
// DD and rotated back, sigma_g = R^T sigma_l R, u_g = R^T u_l (R row-major,
// local = R global).  The reference's BigWhamIO has no working 3DR0
// observation kernel (BieElastostatic<Rectangle<0>, Point<3>, T | W> return
// zeros, bie_elastostatic_rectangle_0_influence.h:222-245); the output
// layout is the one its 3D observation kernels use
// (bie_elastostatic_triangle_0_influence.h:196-215): s11, s22, s33, s12,
// s13, s23 and u1, u2, u3.
#pragma once

#include "bw_r0.h"

namespace bw {
namespace r0 {

// Element data a field evaluation reads: collocation point (3), rotation
// row-major (9), half sides a, b; then the local DD (3).
constexpr int kFieldDoubles = 17;

// el: kFieldDoubles values as above; acc += the 9 field values at p.
BW_HD void add_point_fields(const double *el, const double *p, double G, double nu, double acc[9]) {
  const double *cp = el, *R = el + 3, *dd = el + 14;
  const double a = el[12], b = el[13];
  double d[3], l[3];
  for (int k = 0; k < 3; k++) d[k] = p[k] - cp[k];
  for (int i = 0; i < 3; i++) l[i] = R[3 * i] * d[0] + R[3 * i + 1] * d[1] + R[3 * i + 2] * d[2];
  const Derivs D = derivs(l[0], l[1], l[2], a, b);
  double s[3][6], u[3][3];
  stress_from(D, l[2], G, nu, s);
  displacement_from(D, l[2], nu, u);
  double c[6];  // local stress: xx, yy, zz, xy, xz, yz
  for (int q = 0; q < 6; q++) c[q] = s[0][q] * dd[0] + s[1][q] * dd[1] + s[2][q] * dd[2];
  const double S[3][3] = {{c[0], c[3], c[4]}, {c[3], c[1], c[5]}, {c[4], c[5], c[2]}};
  double T[3][3];  // S R
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) T[i][j] = S[i][0] * R[j] + S[i][1] * R[3 + j] + S[i][2] * R[6 + j];
  auto g = [&](int i, int j) { return R[i] * T[0][j] + R[3 + i] * T[1][j] + R[6 + i] * T[2][j]; };  // (R^T S R)_ij
  acc[0] += g(0, 0);
  acc[1] += g(1, 1);
  acc[2] += g(2, 2);
  acc[3] += g(0, 1);
  acc[4] += g(0, 2);
  acc[5] += g(1, 2);
  double ul[3];
  for (int i = 0; i < 3; i++) ul[i] = u[i][0] * dd[0] + u[i][1] * dd[1] + u[i][2] * dd[2];
  for (int i = 0; i < 3; i++) acc[6 + i] += R[i] * ul[0] + R[3 + i] * ul[1] + R[6 + i] * ul[2];
}

}  // namespace r0
}  // namespace bw
