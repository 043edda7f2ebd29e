// Fields of a straight segment carrying a constant displacement discontinuity
// (the 2DS0 element: plane strain, full space), host and device.
//
// Published solution: Crouch & Starfield, "Boundary Element Methods in Solid
// Mechanics" (1983), section 5.2.  For a segment |x| <= a on y = 0 with DD
// (Dx, Dy) (shear, normal) and
//   f(x, y) = -c [ y (atan2(y, x - a) - atan2(y, x + a))
//                  - (x - a) ln r1 + (x + a) ln r2 ],   c = 1 / (4 pi (1 - nu)),
// r1^2 = (x - a)^2 + y^2, r2^2 = (x + a)^2 + y^2, the displacements and stresses
// are linear in the derivatives of f:
//   ux  = Dx [2(1 - nu) f_y - y f_xx] + Dy [-(1 - 2nu) f_x - y f_xy]
//   uy  = Dx [(1 - 2nu) f_x - y f_xy] + Dy [2(1 - nu) f_y - y f_yy]
//   sxx = 2G Dx [2 f_xy + y f_xyy] + 2G Dy [f_yy + y f_yyy]
//   syy = 2G Dx [-y f_xyy]         + 2G Dy [f_yy - y f_yyy]
//   sxy = 2G Dx [f_yy + y f_yyy]   + 2G Dy [-y f_xyy]
// This is the element of the reference's 2DS0-H kernel (its own closed forms
// are written for the unit segment: We_segment_0 / Se_segment_0,
// src/elasticity/fullspace_iso_2d_segment/elastic_2dP0_segment.cc:82-211); the
// stresses agree with its observation kernel W (bie_elastostatic_segment_0_
// influence.h:320-372).  On the element's own line (y = 0, |x| < a) the
// displacement jumps; like the reference, y = 0 is taken as the limit from
// below (y -> 0-).
//
// Frames (src/elements/segment.h:40-90): t = (v1 - v0) / |v1 - v0|, n = (-t_y,
// t_x); local = R global with R's rows t, n; a stress tensor maps back as
// R^T S R and a vector as R^T u.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define BW_S0_HD __host__ __device__ __forceinline__
#else
#define BW_S0_HD inline
#endif

namespace bw {
namespace s0 {

// One element: centre, half length, unit tangent.
constexpr int kRecordDoubles = 5;  // cx, cy, a, tx, ty
constexpr double kPi = 3.14159265358979323846;

struct Derivs {
  double fx, fy, fxy, fyy, fxyy, fyyy;  // f_xx = -f_yy
};

BW_S0_HD Derivs derivs(double x, double y, double a, double nu) {
  const double c = 1.0 / (4.0 * kPi * (1.0 - nu));
  const double xm = x - a, xp = x + a, y2 = y * y;
  const double r1 = xm * xm + y2, r2 = xp * xp + y2;
  const double ys = (y == 0.0) ? -0.0 : y;  // on the line: the limit from below
  Derivs d;
  d.fx = 0.5 * c * (log(r1) - log(r2));
  d.fy = -c * (atan2(ys, xm) - atan2(ys, xp));
  d.fxy = c * (y / r1 - y / r2);
  d.fyy = -c * (xm / r1 - xp / r2);
  d.fxyy = c * ((xm * xm - y2) / (r1 * r1) - (xp * xp - y2) / (r2 * r2));
  d.fyyy = 2.0 * c * y * (xm / (r1 * r1) - xp / (r2 * r2));
  return d;
}

// Local fields of unit DDs: s[k] = (sxx, syy, sxy), u[k] = (ux, uy) for the DD
// k = 0 (shear, along t) and k = 1 (normal, along n).
BW_S0_HD void local_fields(double x, double y, double a, double G, double nu, double s[2][3], double u[2][2]) {
  const Derivs d = derivs(x, y, a, nu);
  const double fxx = -d.fyy;
  s[0][0] = 2.0 * G * (2.0 * d.fxy + y * d.fxyy);
  s[0][1] = 2.0 * G * (-y * d.fxyy);
  s[0][2] = 2.0 * G * (d.fyy + y * d.fyyy);
  s[1][0] = 2.0 * G * (d.fyy + y * d.fyyy);
  s[1][1] = 2.0 * G * (d.fyy - y * d.fyyy);
  s[1][2] = 2.0 * G * (-y * d.fxyy);
  u[0][0] = 2.0 * (1.0 - nu) * d.fy - y * fxx;
  u[0][1] = (1.0 - 2.0 * nu) * d.fx - y * d.fxy;
  u[1][0] = -(1.0 - 2.0 * nu) * d.fx - y * d.fxy;
  u[1][1] = 2.0 * (1.0 - nu) * d.fy - y * d.fyy;
}

// Global stress (s11, s22, s12) and displacement (u1, u2) at point (px, py)
// due to the element `rec` carrying the local DD (dd_s, dd_n); added to acc
// (5 values: s11, s22, s12, u1, u2).
BW_S0_HD void add_point_fields(const double *rec, double dd_s, double dd_n, double px, double py, double G,
                               double nu, double acc[5]) {
  const double cx = rec[0], cy = rec[1], a = rec[2], tx = rec[3], ty = rec[4];
  const double nx = -ty, ny = tx;
  const double dx = px - cx, dy = py - cy;
  const double xl = tx * dx + ty * dy, yl = nx * dx + ny * dy;
  double s[2][3], u[2][2];
  local_fields(xl, yl, a, G, nu, s, u);
  const double sxx = s[0][0] * dd_s + s[1][0] * dd_n;
  const double syy = s[0][1] * dd_s + s[1][1] * dd_n;
  const double sxy = s[0][2] * dd_s + s[1][2] * dd_n;
  const double ux = u[0][0] * dd_s + u[1][0] * dd_n;
  const double uy = u[0][1] * dd_s + u[1][1] * dd_n;
  // R^T S R = sxx t t^T + syy n n^T + sxy (t n^T + n t^T); R^T u = ux t + uy n
  acc[0] += sxx * tx * tx + syy * nx * nx + 2.0 * sxy * tx * nx;
  acc[1] += sxx * ty * ty + syy * ny * ny + 2.0 * sxy * ty * ny;
  acc[2] += sxx * tx * ty + syy * nx * ny + sxy * (tx * ny + nx * ty);
  acc[3] += ux * tx + uy * nx;
  acc[4] += ux * ty + uy * ny;
}

// Hypersingular (H) entry between two elements: tractions at the receiver's
// centre, in the receiver's frame (shear along its tangent, normal along its
// normal), due to unit local DDs of the source; K[j][k] = traction j due to
// DD k.  The reference's BieElastostatic<Segment<0>, Segment<0>, H>
// (bie_elastostatic_segment_0_influence.h:176-232) stores the same 2 x 2
// block column-major.
BW_S0_HD void h_entry(const double *src, const double *rcv, double G, double nu, double K[2][2]) {
  const double tx = rcv[3], ty = rcv[4], nx = -ty, ny = tx;
  for (int k = 0; k < 2; k++) {
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    add_point_fields(src, k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, rcv[0], rcv[1], G, nu, acc);
    const double t1 = acc[0] * nx + acc[2] * ny, t2 = acc[2] * nx + acc[1] * ny;  // sigma n
    K[0][k] = t1 * tx + t2 * ty;
    K[1][k] = t1 * nx + t2 * ny;
  }
}

}  // namespace s0
}  // namespace bw
