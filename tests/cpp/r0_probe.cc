// Host build of bigwham_dev_b200/csrc/bw_r0.h for tests/test_r0_kernel_cpu.py:
// the same functions the device code uses, exported with C linkage.
#include "bw_r0.h"

extern "C" {

void probe_r0_stress(double x, double y, double z, double a, double b, double G, double nu, double *out) {
  double s[3][6];
  bw::r0::stress(x, y, z, a, b, G, nu, s);
  for (int i = 0; i < 3; i++)
    for (int c = 0; c < 6; c++) out[6 * i + c] = s[i][c];
}

void probe_r0_displacement(double x, double y, double z, double a, double b, double nu, double *out) {
  double u[3][3];
  bw::r0::displacement(x, y, z, a, b, nu, u);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) out[3 * i + j] = u[i][j];
}

void probe_r0_influence(const double *frame_s, double a_s, double b_s, const double *frame_r, double G, double nu,
                        double *out) {
  // frame: collocation point (3), row-major rotation (9), normal (3)
  double K[3][3];
  bw::r0::influence_h(frame_s, frame_s + 3, a_s, b_s, frame_r, frame_r + 3, frame_r + 12, G, nu, K);
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) out[3 * j + i] = K[j][i];
}

}  // extern "C"
