// Rectangular displacement-discontinuity element (BigWham's 3DR0 kernel
// family): stresses and displacements at a point, for host and device code.
//
// A rectangle [-a, a] x [-b, b] in the plane z = 0 of its local frame carries
// a uniform displacement discontinuity (Dx, Dy, Dz).  With
//   I(x, y, z) = int_{-a}^{a} int_{-b}^{b} dxi deta / R,
//   R = sqrt((x - xi)^2 + (y - eta)^2 + z^2),
// the Kelvin solution integrated over the rectangle gives, with
// C = G / (4 pi (1 - nu)) and derivatives of I written I_x, I_xz, ...:
//   DD x: sxx = C (2 I_xz - z I_xxx)          syy = C (2 nu I_xz - z I_xyy)
//         szz = -C z I_xzz                     sxy = C ((1 - nu) I_yz - z I_xxy)
//         sxz = C (I_zz + nu I_yy - z I_xxz)   syz = -C (nu I_xy + z I_xyz)
//   DD y: x <-> y in the DD x row
//   DD z: sxx = C (I_zz + (1 - 2 nu) I_yy - z I_xxz)
//         syy = C (I_zz + (1 - 2 nu) I_xx - z I_yyz)
//         szz = C (I_zz - z I_zzz)              sxy = -C ((1 - 2 nu) I_xy + z I_xyz)
//         sxz = -C z I_xzz                      syz = -C z I_yzz
// and displacements, with c = 1 / (8 pi (1 - nu)), u_i due to DD j:
//   u_x = c [Dx (2(1 - nu) I_z - z I_xx) - Dy z I_xy - Dz ((1 - 2 nu) I_x + z I_xz)]
//   u_y = c [-Dx z I_xy + Dy (2(1 - nu) I_z - z I_yy) - Dz ((1 - 2 nu) I_y + z I_yz)]
//   u_z = c [Dx ((1 - 2 nu) I_x - z I_xz) + Dy ((1 - 2 nu) I_y - z I_yz)
//            + Dz (2(1 - nu) I_z - z I_zz)]
// These follow from the Kelvin Green's function written as
// G_pk = [4 (1 - nu) delta_pk / R - R_,pk] / (16 pi G (1 - nu)) and Volterra's
// formula for a discontinuity across a plane; they are the conventions of the
// reference's StressesKernelR0 / DisplacementKernelR0
// (src/elasticity/fullspace_iso_3d_rectangle/elastic_3dR0_element.h), which
// this header restates.
//
// I and its derivatives are signed corner sums sum_{sx, sy} sx sy f(X, Y, z),
// X = x + sx a, Y = y + sy b, of the antiderivative
//   F = X ln(Y + R) + Y ln(X + R) - z atan(X Y / (z R))
// (d^2 F / dX dY = 1 / R) and its derivatives, each written up to terms in X
// alone or Y alone, which cancel in the sum:
//   F_x = ln(Y + R)       F_xx = X / (R (R + Y))     F_xy = 1 / R
//   F_z = -atan(X Y / (z R))                         F_xz = z / (R (R + Y))
//   F_zz = X Y (X^2 + Y^2 + 2 z^2) / (R (X^2 + z^2) (Y^2 + z^2))
//   F_xxy = -X / R^3      F_xyz = -z / R^3
//   F_xxx = d/dX F_xx     F_xxz = d/dz F_xx          F_xzz = d/dz F_xz
// (y forms by X <-> Y), and I_zzz = -(I_xxz + I_yyz) (I is harmonic off the
// plane).  Numerics:
// * R + Y cancels when Y < 0 and X^2 + z^2 << Y^2, so it is evaluated as
//   (X^2 + z^2) / (R - Y) there (an identity);
// * in the element plane (z == 0) I_xz = I_yz = 0, I_zz = -(I_xx + I_yy),
//   and the z-weighted terms vanish.  When both corners on one side of the
//   rectangle have Y < 0 (the point lies beyond it in y) their I_x and I_xx
//   terms are combined analytically, which stays finite on the edge's line
//   (X = 0); likewise in x.  Points on an edge itself are singular.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define BW_HD __host__ __device__ __forceinline__
#else
#define BW_HD inline
#endif

namespace bw {
namespace r0 {

// Derivatives of I; index names as in the formulas above.
struct Derivs {
  double x, y, z;
  double xx, yy, zz, xy, xz, yz;
  double xxx, yyy, zzz, xxy, xyy, xxz, yyz, xzz, yzz, xyz;
};

constexpr double kPi = 3.14159265358979323846;

// R + Y without cancellation (q = X^2 + z^2).
BW_HD double r_plus(double R, double Y, double q) { return Y >= 0.0 ? R + Y : q / (R - Y); }

// Off the element plane (z != 0): every derivative up to third order.
BW_HD Derivs derivs_offplane(double x, double y, double z, double a, double b) {
  Derivs d = {};
  for (int cx = 0; cx < 2; cx++) {
    for (int cy = 0; cy < 2; cy++) {
      const double sx = cx ? -1.0 : 1.0, sy = cy ? -1.0 : 1.0, s = sx * sy;
      const double X = x + sx * a, Y = y + sy * b;
      const double X2 = X * X, Y2 = Y * Y, z2 = z * z;
      const double R = sqrt(X2 + Y2 + z2), R2 = R * R, R3 = R2 * R;
      const double qx = X2 + z2, qy = Y2 + z2;
      const double RY = r_plus(R, Y, qx), RX = r_plus(R, X, qy);
      d.x += s * log(RY);
      d.y += s * log(RX);
      d.z -= s * atan(X * Y / (z * R));
      d.xx += s * X / (R * RY);
      d.yy += s * Y / (R * RX);
      d.xy += s / R;
      d.xz += s * z / (R * RY);
      d.yz += s * z / (R * RX);
      d.zz += s * X * Y * (X2 + Y2 + 2.0 * z2) / (R * qx * qy);
      d.xxy -= s * X / R3;
      d.xyy -= s * Y / R3;
      d.xyz -= s * z / R3;
      const double RY2 = RY * RY, RX2 = RX * RX;
      d.xxx += s * (R * RY - X2 * (2.0 * R + Y) / R) / (R2 * RY2);
      d.yyy += s * (R * RX - Y2 * (2.0 * R + X) / R) / (R2 * RX2);
      d.xxz -= s * X * z * (2.0 * R + Y) / (R3 * RY2);
      d.yyz -= s * Y * z * (2.0 * R + X) / (R3 * RX2);
      d.xzz += s * (R * RY - z2 * (2.0 * R + Y) / R) / (R2 * RY2);
      d.yzz += s * (R * RX - z2 * (2.0 * R + X) / R) / (R2 * RX2);
    }
  }
  d.zzz = -(d.xxz + d.yyz);
  return d;
}

// Sum over the two corners of one side (coordinate P fixed; Q1 = q - w,
// Q2 = q + w the other coordinate at the two corners, signs -1 / +1) of
// ln(Q + R) and of P / (R (R + Q)), in the plane z = 0.
struct PairSums {
  double ln, first;
};

BW_HD PairSums pair_inplane(double P, double q, double w) {
  const double Q1 = q - w, Q2 = q + w;
  const double R1 = sqrt(P * P + Q1 * Q1), R2 = sqrt(P * P + Q2 * Q2);
  PairSums r;
  if (Q2 < 0.0) {
    // both corners beyond the side: ln(Q + R) = ln(P^2) - ln(R - Q), the
    // ln(P^2) parts cancel; P / (R (R + Q)) = 1 / P - Q / (R P), the 1 / P
    // parts cancel, and the rest is written without 0 / 0 at P = 0.
    r.ln = log(R1 - Q1) - log(R2 - Q2);
    const double t1 = P * P / (Q1 * Q1), t2 = P * P / (Q2 * Q2);
    const double r1 = sqrt(1.0 + t1), r2 = sqrt(1.0 + t2);
    r.first = P * (4.0 * w * q / (Q1 * Q1 * Q2 * Q2)) / (r1 * r2 * (r1 + r2));
  } else {
    const double q2 = P * P;
    const double RQ1 = r_plus(R1, Q1, q2), RQ2 = r_plus(R2, Q2, q2);
    r.ln = log(RQ2) - log(RQ1);
    r.first = P / (R2 * RQ2) - P / (R1 * RQ1);
  }
  return r;
}

// In the element plane (z == 0): I_x, I_y, I_xx, I_yy, I_xy, I_zz and the
// one-sided I_z (limit from z > 0); the rest is zero there.
BW_HD Derivs derivs_inplane(double x, double y, double a, double b) {
  Derivs d = {};
  for (int cx = 0; cx < 2; cx++) {
    const double sx = cx ? -1.0 : 1.0;
    const PairSums p = pair_inplane(x + sx * a, y, b);
    d.x += sx * p.ln;
    d.xx += sx * p.first;
  }
  for (int cy = 0; cy < 2; cy++) {
    const double sy = cy ? -1.0 : 1.0;
    const PairSums p = pair_inplane(y + sy * b, x, a);
    d.y += sy * p.ln;
    d.yy += sy * p.first;
  }
  for (int cx = 0; cx < 2; cx++)
    for (int cy = 0; cy < 2; cy++) {
      const double sx = cx ? -1.0 : 1.0, sy = cy ? -1.0 : 1.0, s = sx * sy;
      const double X = x + sx * a, Y = y + sy * b;
      d.xy += s / sqrt(X * X + Y * Y);
      // -atan(X Y / (z R)) as z -> 0+
      const double sg = (X * Y > 0.0) ? 1.0 : (X * Y < 0.0 ? -1.0 : 0.0);
      d.z -= s * sg * (0.5 * kPi);
    }
  d.zz = -(d.xx + d.yy);
  return d;
}

BW_HD Derivs derivs(double x, double y, double z, double a, double b) {
  return z == 0.0 ? derivs_inplane(x, y, a, b) : derivs_offplane(x, y, z, a, b);
}

// Stresses in the element's local frame: s[dd][c], dd = DD x, y, z and
// c = xx, yy, zz, xy, xz, yz (the reference's StressesKernelR0 layout), from
// the derivatives at (x, y, z); stress() evaluates them first.
BW_HD void stress_from(const Derivs &D, double z, double G, double nu, double s[3][6]) {
  const double C = G / (4.0 * kPi * (1.0 - nu));
  s[0][0] = C * (2.0 * D.xz - z * D.xxx);
  s[0][1] = C * (2.0 * nu * D.xz - z * D.xyy);
  s[0][2] = -C * z * D.xzz;
  s[0][3] = C * ((1.0 - nu) * D.yz - z * D.xxy);
  s[0][4] = C * (D.zz + nu * D.yy - z * D.xxz);
  s[0][5] = -C * (nu * D.xy + z * D.xyz);
  s[1][0] = C * (2.0 * nu * D.yz - z * D.xxy);
  s[1][1] = C * (2.0 * D.yz - z * D.yyy);
  s[1][2] = -C * z * D.yzz;
  s[1][3] = C * ((1.0 - nu) * D.xz - z * D.xyy);
  s[1][4] = -C * (nu * D.xy + z * D.xyz);
  s[1][5] = C * (D.zz + nu * D.xx - z * D.yyz);
  s[2][0] = C * (D.zz + (1.0 - 2.0 * nu) * D.yy - z * D.xxz);
  s[2][1] = C * (D.zz + (1.0 - 2.0 * nu) * D.xx - z * D.yyz);
  s[2][2] = C * (D.zz - z * D.zzz);
  s[2][3] = -C * ((1.0 - 2.0 * nu) * D.xy + z * D.xyz);
  s[2][4] = -C * z * D.xzz;
  s[2][5] = -C * z * D.yzz;
}

BW_HD void stress(double x, double y, double z, double a, double b, double G, double nu, double s[3][6]) {
  stress_from(derivs(x, y, z, a, b), z, G, nu, s);
}

// Displacements in the element's local frame: u[i][j] = component i due to
// unit DD j (the reference's DisplacementKernelR0 layout), from the
// derivatives; displacement() evaluates them first.
BW_HD void displacement_from(const Derivs &D, double z, double nu, double u[3][3]) {
  const double c = 1.0 / (8.0 * kPi * (1.0 - nu)), k1 = 2.0 * (1.0 - nu), k2 = 1.0 - 2.0 * nu;
  u[0][0] = c * (k1 * D.z - z * D.xx);
  u[1][0] = -c * z * D.xy;
  u[2][0] = c * (k2 * D.x - z * D.xz);
  u[0][1] = -c * z * D.xy;
  u[1][1] = c * (k1 * D.z - z * D.yy);
  u[2][1] = c * (k2 * D.y - z * D.yz);
  u[0][2] = -c * (k2 * D.x + z * D.xz);
  u[1][2] = -c * (k2 * D.y + z * D.yz);
  u[2][2] = c * (k1 * D.z - z * D.zz);
}

BW_HD void displacement(double x, double y, double z, double a, double b, double nu, double u[3][3]) {
  displacement_from(derivs(x, y, z, a, b), z, nu, u);
}

// Hypersingular (H) kernel entry between two rectangles: tractions at the
// receiver's collocation point, in the receiver's local frame, due to unit
// DDs of the source in the source's local frame; K[j][i] = traction j due to
// DD i.  Frames as BigWham's elements hold them: rot is row-major with
// local = rot * global; cp the collocation point (centroid), n_r the
// receiver's unit normal, (a_s, b_s) the source's half sides along its local
// x and y.  The steps are those of the reference's
// BieElastostatic<Rectangle<0>, Rectangle<0>, H>::influence
// (src/elasticity/fullspace_iso_3d_rectangle/
// bie_elastostatic_rectangle_0_influence.h:29-125): stresses at the receiver
// point in the source frame, traction on the receiver normal, rotated to
// global and then to the receiver frame.
BW_HD void influence_h(const double *cp_s, const double *rot_s, double a_s, double b_s, const double *cp_r,
                       const double *rot_r, const double *n_r, double G, double nu, double K[3][3]) {
  double d[3], dl[3], nl[3];
  for (int k = 0; k < 3; k++) d[k] = cp_r[k] - cp_s[k];
  for (int r = 0; r < 3; r++) {
    dl[r] = rot_s[3 * r] * d[0] + rot_s[3 * r + 1] * d[1] + rot_s[3 * r + 2] * d[2];
    nl[r] = rot_s[3 * r] * n_r[0] + rot_s[3 * r + 1] * n_r[1] + rot_s[3 * r + 2] * n_r[2];
  }
  double s[3][6];
  stress(dl[0], dl[1], dl[2], a_s, b_s, G, nu, s);
  for (int i = 0; i < 3; i++) {
    // traction on nl in the source frame (symmetric tensor xx yy zz xy xz yz)
    const double t0 = s[i][0] * nl[0] + s[i][3] * nl[1] + s[i][4] * nl[2];
    const double t1 = s[i][3] * nl[0] + s[i][1] * nl[1] + s[i][5] * nl[2];
    const double t2 = s[i][4] * nl[0] + s[i][5] * nl[1] + s[i][2] * nl[2];
    // to global (rot_s^T) and to the receiver frame (rot_r)
    double g[3];
    for (int k = 0; k < 3; k++) g[k] = rot_s[k] * t0 + rot_s[3 + k] * t1 + rot_s[6 + k] * t2;
    for (int j = 0; j < 3; j++) K[j][i] = rot_r[3 * j] * g[0] + rot_r[3 * j + 1] * g[1] + rot_r[3 * j + 2] * g[2];
  }
}

// Element record used by the assembly: collocation point (3), rotation
// row-major (9), unit normal (3), half sides a, b.
constexpr int kFrameDoubles = 17;

// The 3 x 3 H-kernel entry of receiver element `rec` and source element
// `src` (records as above), written column-major into a full-rank block of
// leading dimension ld at (row0, col0): out[(col0 + i) * ld + row0 + j] =
// traction j at the receiver due to DD i of the source.
BW_HD void h_entry_into_block(const double *src, const double *rec, double G, double nu, double *out, long long ld,
                              long long row0, long long col0) {
  double K[3][3];
  influence_h(src, src + 3, src[15], src[16], rec, rec + 3, rec + 12, G, nu, K);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) out[(col0 + i) * ld + row0 + j] = K[j][i];
}

}  // namespace r0
}  // namespace bw
