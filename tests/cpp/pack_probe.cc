// Run-based packing (bigwham_dev_b200/csrc/bw_pack.h, the device packer's
// element copy) against the host fill (bw::fill_items) on a real plan built by
// the layout library, byte for byte; used by tests/test_pack_cpu.py.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bw_layout.h"
#include "bw_pack.h"

extern "C" int probe_pack_compare(int dof, long long n_rows, long long n_cols, long long n_fr, const long long *fr,
                                  const double *fr_data, long long fr_len, long long n_lr, const long long *lr,
                                  const double *lr_data, long long lr_len, long long *diff_bytes, long long *runs) {
  try {
    bw::Problem p;
    p.dof = dof;
    p.n_rows = n_rows;
    p.n_cols = n_cols;
    long long o = 0;
    for (long long k = 0; k < n_fr; k++) {
      const long long m = (fr[4 * k + 2] - fr[4 * k]) * dof, n = (fr[4 * k + 3] - fr[4 * k + 1]) * dof;
      p.fr.push_back({fr[4 * k] * dof, fr[4 * k + 1] * dof, m, n, bw::View{fr_data + o, m, false}});
      o += m * n;
    }
    o = 0;
    for (long long k = 0; k < n_lr; k++) {
      const long long m = (lr[5 * k + 2] - lr[5 * k]) * dof, n = (lr[5 * k + 3] - lr[5 * k + 1]) * dof,
                      r = lr[5 * k + 4];
      p.lr.push_back({lr[5 * k] * dof, lr[5 * k + 1] * dof, m, n, r, bw::View{lr_data + o, m > 0 ? m : 1, false},
                      bw::View{lr_data + o + m * r, r > 0 ? r : 1, false}});
      o += r * (m + n);
    }
    // per stored block maxima, as a device reduction would compute them
    std::vector<double> mfr(p.fr.size()), ma(p.lr.size()), mb(p.lr.size());
    std::vector<int> bfr(p.fr.size(), 0), blr(p.lr.size(), 0);
    auto mx = [](const bw::View &v, long long m, long long n, int &bad) {
      double s = 0.0;
      for (long long j = 0; j < n; j++)
        for (long long i = 0; i < m; i++) {
          const double a = std::fabs(v.at(i, j));
          if (!(a <= 1.0e300)) bad = 1;
          s = std::max(s, a);
        }
      return s;
    };
    for (size_t k = 0; k < p.fr.size(); k++) mfr[k] = mx(p.fr[k].a, p.fr[k].m, p.fr[k].n, bfr[k]);
    for (size_t k = 0; k < p.lr.size(); k++) {
      ma[k] = mx(p.lr[k].A, p.lr[k].m, p.lr[k].r, blr[k]);
      mb[k] = mx(p.lr[k].B, p.lr[k].r, p.lr[k].n, blr[k]);
    }
    int q = 0;
    for (int tr = 0; tr < 2; tr++) {
      bw::OperatorPlan op;
      bw::build_operator(p, tr == 1, 148, op);
      bw::compute_scales(p, tr == 1, true, op);
      {
        bw::OperatorPlan op2 = op;
        bw::scales_from_maxima(p, tr == 1, true, mfr.data(), ma.data(), mb.data(), bfr.data(), blr.data(), op2);
        if (op2.scale_fr != op.scale_fr || op2.scale_a != op.scale_a || op2.scale_b != op.scale_b ||
            op2.t_scale != op.t_scale)
          return 2;
      }
      for (int prec = 0; prec < 3; prec++) bw::build_chunks(p, tr == 1, prec, 148, op);
      for (int phase = 0; phase < 2; phase++)
        for (int prec = 0; prec < 3; prec++, q++) {
          const int es = bw::esize_of(prec);
          const size_t bytes = (size_t)op.ph[phase].n_elems[prec] * es;
          std::vector<unsigned char> a(bytes, 0), b(bytes, 0);
          bw::fill_items(p, tr == 1, op, phase, prec, 0, (int64_t)op.ph[phase].items.size(), 0, a.data());
          std::vector<bw::PackRun> rv;
          bw::build_pack_runs(p, tr == 1, op, phase, prec, fr_data, fr_len, lr_data, lr_len, rv);
          if (prec == 0) bw::pack::runs_host<0>(b.data(), rv.data(), (int64_t)rv.size(), fr_data, lr_data);
          if (prec == 1) bw::pack::runs_host<1>(b.data(), rv.data(), (int64_t)rv.size(), fr_data, lr_data);
          if (prec == 2) bw::pack::runs_host<2>(b.data(), rv.data(), (int64_t)rv.size(), fr_data, lr_data);
          long long d = 0;
          for (size_t k = 0; k < bytes; k++) d += a[k] != b[k];
          diff_bytes[q] = d;
          runs[q] = (long long)rv.size();
        }
    }
    return 0;
  } catch (...) {
    return 1;
  }
}
