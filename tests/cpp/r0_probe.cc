// Host build of bigwham_dev_b200/csrc/bw_r0.h for tests/test_r0_kernel_cpu.py:
// the same functions the device code uses, exported with C linkage.
#include "bw_aca.h"
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

// Full-rank blocks of a 3DR0-H H-matrix assembled on the host with the same
// entry function as the device kernel: fr (n_fr x 4, permuted points), perm
// (permuted point -> element), frames (n_elems x 17); out: the blocks back to
// back, column-major.
void probe_r0_fr_blocks(const double *frames, double G, double nu, long long n_fr, const long long *fr,
                        const long long *perm, double *out) {
  long long off = 0;
  for (long long k = 0; k < n_fr; k++) {
    const long long i0 = fr[4 * k], j0 = fr[4 * k + 1], mp = fr[4 * k + 2] - i0, np_ = fr[4 * k + 3] - j0;
    for (long long jj = 0; jj < np_; jj++)
      for (long long ii = 0; ii < mp; ii++)
        bw::r0::h_entry_into_block(frames + bw::r0::kFrameDoubles * perm[j0 + jj],
                                   frames + bw::r0::kFrameDoubles * perm[i0 + ii], G, nu, out + off, 3 * mp, 3 * ii,
                                   3 * jj);
    off += 9 * mp * np_;
  }
}

// Block ACA of the low-rank block (rows [i0, i1), columns [j0, j1) in
// permuted points) of a 3DR0-H H-matrix, with the entry function of the
// device assembly.  A: (i1 - i0) 3 x cap 3, B: cap 3 x (j1 - j0) 3,
// column-major; returns the rank in blocks (-1 when cap was too small).
int probe_r0_aca(const double *frames, double G, double nu, const long long *perm, long long i0, long long j0,
                 long long i1, long long j1, double eps, int cap, double *A, double *B, double *err) {
  const int n0 = (int)(i1 - i0), n1 = (int)(j1 - j0);
  double *work = new double[(size_t)(n0 + n1) * 9 + n0 + n1];
  auto entry = [&](int i, int j, double K[3][3]) {
    bw::r0::influence_h(frames + bw::r0::kFrameDoubles * perm[j0 + j], frames + bw::r0::kFrameDoubles * perm[j0 + j] + 3,
                        frames[bw::r0::kFrameDoubles * perm[j0 + j] + 15], frames[bw::r0::kFrameDoubles * perm[j0 + j] + 16],
                        frames + bw::r0::kFrameDoubles * perm[i0 + i], frames + bw::r0::kFrameDoubles * perm[i0 + i] + 3,
                        frames + bw::r0::kFrameDoubles * perm[i0 + i] + 12, G, nu, K);
  };
  const bw::aca::Result r = bw::aca::block_aca_host(entry, n0, n1, eps, cap, A, B, work);
  delete[] work;
  *err = r.error;
  return r.overflow ? -1 : r.rank_blocks;
}

}  // extern "C"
