// Host-side layout builder (see bw_layout.h for the scheme).
#include "bw_layout.h"

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <queue>
#include <stdexcept>
#include <string>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace bw {

int esize_of(int prec) { return prec == 0 ? 8 : (prec == 1 ? 4 : 2); }

// Round-to-nearest-even FP32 -> BF16 on the bit pattern (NaN kept quiet).
uint16_t to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return static_cast<uint16_t>((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return static_cast<uint16_t>(u >> 16);
}

float from_bf16(uint16_t b) {
  uint32_t u = static_cast<uint32_t>(b) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

namespace {

// Offsets, counts and row indices of the plan are 32-bit fields the kernels
// read; a problem whose layout outgrows them is refused instead of wrapping.
int32_t i32(int64_t v, const char *what) {
  if (v < INT32_MIN || v > INT32_MAX)
    throw std::length_error(std::string("layout field ") + what + " exceeds 32 bits (" + std::to_string(v) + ")");
  return static_cast<int32_t>(v);
}

uint32_t u31(int64_t v, const char *what) {
  if (v < 0 || v > 0x7fffffffLL)
    throw std::length_error(std::string("layout field ") + what + " exceeds 31 bits (" + std::to_string(v) + ")");
  return static_cast<uint32_t>(v);
}

// The blocks of the operator being laid out: H itself, or H^T built from the
// same storage (FR: A^T; LR: (A B)^T = B^T A^T, i.e. A' = B^T and B' = A^T).
struct EffFull {
  int64_t i0, j0, m, n;
  View a;
};
struct EffLow {
  int64_t i0, j0, m, n, r;
  View A, B;
};

View flip(View v) {
  v.trans = !v.trans;
  return v;
}

EffFull eff_full(const Problem &p, bool tr, size_t k) {
  const FullBlock &b = p.fr[k];
  if (!tr) return {b.i0, b.j0, b.m, b.n, b.a};
  return {b.j0, b.i0, b.n, b.m, flip(b.a)};
}

EffLow eff_low(const Problem &p, bool tr, size_t k) {
  const LowRankBlock &b = p.lr[k];
  if (!tr) return {b.i0, b.j0, b.m, b.n, b.r, b.A, b.B};
  return {b.j0, b.i0, b.n, b.m, b.r, flip(b.B), flip(b.A)};
}

[[noreturn]] void fail(const std::string &msg) { throw std::runtime_error(msg); }

int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

}  // namespace

void build_operator(const Problem &p, bool tr, int grid, OperatorPlan &op) {
  const int64_t n_out = tr ? p.n_cols : p.n_rows;
  const int64_t n_in = tr ? p.n_rows : p.n_cols;
  op = OperatorPlan{};
  op.n_out = n_out;
  op.n_in = n_in;
  const size_t nfr = p.fr.size(), nlr = p.lr.size();

  // ---- range checks
  for (size_t k = 0; k < nfr; k++) {
    const FullBlock &b = p.fr[k];
    if (b.m <= 0 || b.n <= 0 || b.i0 < 0 || b.j0 < 0 || b.i0 + b.m > p.n_rows || b.j0 + b.n > p.n_cols)
      fail("full block " + std::to_string(k) + " out of range");
    if (!b.a.p || b.a.ld < b.m) fail("full block " + std::to_string(k) + ": null data or lda < m");
  }
  for (size_t k = 0; k < nlr; k++) {
    const LowRankBlock &b = p.lr[k];
    if (b.m <= 0 || b.n <= 0 || b.r < 0 || b.i0 < 0 || b.j0 < 0 || b.i0 + b.m > p.n_rows ||
        b.j0 + b.n > p.n_cols)
      fail("low-rank block " + std::to_string(k) + " out of range");
    if (b.r > 0 && (!b.A.p || !b.B.p || b.A.ld < b.m || b.B.ld < b.r))
      fail("low-rank block " + std::to_string(k) + ": null data or leading dimension too small");
    if (b.r > 65535) fail("low-rank block " + std::to_string(k) + ": rank above 65535");
  }
  if (n_out > INT32_MAX || n_in > INT32_MAX) fail("problem too large for 32-bit offsets");

  // ---- phase 1: B factors stacked per column cluster; t follows stack order
  std::map<std::pair<int64_t, int64_t>, std::vector<int64_t>> stacks;  // (j0, n) -> blocks
  for (size_t k = 0; k < nlr; k++) {
    EffLow b = eff_low(p, tr, k);
    if (b.r > 0) stacks[{b.j0, b.n}].push_back((int64_t)k);
  }
  op.t_off.assign(nlr, 0);
  int64_t t = 0;
  for (auto &kv : stacks)
    for (int64_t k : kv.second) {
      op.t_off[k] = t;
      t += eff_low(p, tr, k).r;
    }
  op.t_len = t;
  if (t > INT32_MAX) fail("sum of ranks above 2^31-1");
  op.n_stacks = (int64_t)stacks.size();
  grid = std::max(1, grid);
  int64_t e1 = 0;  // phase-1 entries
  for (size_t k = 0; k < nlr; k++) e1 += p.lr[k].r * eff_low(p, tr, k).n;
  const int64_t cap1 = std::max<int64_t>(1, e1 / grid / std::max(1, p.tune.items_per_cta[0]));
  PhasePlan &p1 = op.ph[0];
  for (auto &kv : stacks) {
    const int64_t j0 = kv.first.first, n = kv.first.second;
    int64_t R = 0;
    for (int64_t k : kv.second) R += eff_low(p, tr, k).r;
    // equal cuts of at most kHMax rows (fewer when n is wide, so no item holds
    // more than cap1 entries; at least 16 rows), multiples of kRowAlign
    const int64_t rmax = std::min<int64_t>(kHMax, std::max<int64_t>(16, (cap1 / n) / 16 * 16));
    const int64_t nit = (R + rmax - 1) / rmax;
    const int64_t cut = align_up((R + nit - 1) / nit, kRowAlign);
    size_t bi = 0;      // block of the stack
    int64_t br = 0;     // next row inside that block
    for (int64_t r0 = 0; r0 < R; r0 += cut) {
      Item it;
      it.h = i32(std::min<int64_t>(cut, R - r0), "item rows");
      it.hpad = i32(align_up(it.h, kRowAlign), "item rows");
      it.ncols = n;
      it.out_off = i32(op.t_off[kv.second[bi]] + br, "t offset");
      int64_t need = it.h;
      while (need > 0) {
        const int64_t k = kv.second[bi];
        const int64_t rk = eff_low(p, tr, k).r;
        const int64_t take = std::min<int64_t>(need, rk - br);
        it.pieces.push_back({k, br, take});
        need -= take;
        br += take;
        if (br == rk) {
          bi++;
          br = 0;
        }
      }
      it.segs.push_back({2, -1, 0, n, 0, j0});
      p1.items.push_back(std::move(it));
    }
  }

  // batch members along the output and input axes (one member if none given)
  std::vector<int64_t> out_off{0, n_out}, in_off{0, n_in};
  if (!p.row_off.empty()) {
    out_off = tr ? p.col_off : p.row_off;
    in_off = tr ? p.row_off : p.col_off;
  }

  // ---- row panels: finest partition of [0, n_out) by block row boundaries
  // (and member boundaries)
  std::vector<int64_t> bounds(out_off.begin(), out_off.end());
  for (size_t k = 0; k < nfr; k++) {
    EffFull b = eff_full(p, tr, k);
    bounds.push_back(b.i0);
    bounds.push_back(b.i0 + b.m);
  }
  for (size_t k = 0; k < nlr; k++) {
    EffLow b = eff_low(p, tr, k);
    bounds.push_back(b.i0);
    bounds.push_back(b.i0 + b.m);
  }
  std::sort(bounds.begin(), bounds.end());
  bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
  std::vector<int64_t> pb;  // panel starts, with tall panels cut into equal parts of <= kHMax rows
  for (size_t i = 0; i + 1 < bounds.size(); i++) {
    const int64_t H = bounds[i + 1] - bounds[i];
    const int64_t nit = (H + kHMax - 1) / kHMax;
    const int64_t cut = align_up((H + nit - 1) / nit, kRowAlign);
    for (int64_t s = bounds[i]; s < bounds[i + 1]; s += cut) pb.push_back(s);
  }
  pb.push_back(n_out);
  const size_t npan = pb.size() - 1;
  op.n_panels = static_cast<int64_t>(npan);

  // blocks covering each panel (a block covers a contiguous range of panels)
  auto first_panel = [&](int64_t row) {
    return static_cast<size_t>(std::upper_bound(pb.begin(), pb.end(), row) - pb.begin()) - 1;
  };
  struct Cover {
    int kind;  // 0 FR, 1 LR
    int64_t k;
    int64_t j0, n;
  };
  std::vector<std::vector<Cover>> cov(npan);
  for (size_t k = 0; k < nfr; k++) {
    EffFull b = eff_full(p, tr, k);
    for (size_t q = first_panel(b.i0); q < npan && pb[q] < b.i0 + b.m; q++)
      cov[q].push_back({0, (int64_t)k, b.j0, b.n});
  }
  for (size_t k = 0; k < nlr; k++) {
    EffLow b = eff_low(p, tr, k);
    for (size_t q = first_panel(b.i0); q < npan && pb[q] < b.i0 + b.m; q++)
      cov[q].push_back({1, (int64_t)k, b.j0, b.n});
  }
  // coverage: the column intervals of each panel must tile its member's
  // columns [in_off[k], in_off[k+1]) exactly ([0, n_in) for one member)
  for (size_t q = 0; q < npan; q++) {
    auto &c = cov[q];
    std::sort(c.begin(), c.end(), [](const Cover &a, const Cover &b) { return a.j0 < b.j0; });
    const size_t mk = static_cast<size_t>(std::upper_bound(out_off.begin(), out_off.end(), pb[q]) - out_off.begin()) - 1;
    const int64_t lo = in_off[mk], hi = in_off[mk + 1];
    int64_t at = lo;
    for (const Cover &e : c) {
      if (e.j0 < lo || e.j0 + e.n > hi)
        fail("a block in rows [" + std::to_string(pb[q]) + ", " + std::to_string(pb[q + 1]) +
             ") reaches outside its batch member's columns");
      if (e.j0 < at)
        fail("blocks overlap in rows [" + std::to_string(pb[q]) + ", " + std::to_string(pb[q + 1]) + ")");
      if (e.j0 > at)
        fail("columns [" + std::to_string(at) + ", " + std::to_string(e.j0) + ") not covered in rows [" +
             std::to_string(pb[q]) + ", " + std::to_string(pb[q + 1]) + ")");
      at = e.j0 + e.n;
    }
    if (at != hi)
      fail("columns [" + std::to_string(at) + ", " + std::to_string(hi) + ") not covered in rows [" +
           std::to_string(pb[q]) + ", " + std::to_string(pb[q + 1]) + ")");
  }

  // ---- phase 2 items: one per panel (FR slices first: they do not depend on
  // t); panels holding more than cap2 entries are cut into row parts
  PhasePlan &p2 = op.ph[1];
  int64_t e2 = 0;
  std::vector<int64_t> pw(npan, 0);
  for (size_t q = 0; q < npan; q++) {
    for (const Cover &e : cov[q]) pw[q] += e.kind == 0 ? e.n : eff_low(p, tr, e.k).r;
    e2 += pw[q] * (pb[q + 1] - pb[q]);
  }
  const int64_t cap2 = std::max<int64_t>(1, e2 / grid / std::max(1, p.tune.items_per_cta[1]));
  for (size_t q = 0; q < npan; q++) {
    const int64_t H = pb[q + 1] - pb[q];
    int64_t parts = 1;
    if (pw[q] > 0 && H * pw[q] > cap2) parts = std::min<int64_t>((H * pw[q] + cap2 - 1) / cap2, std::max<int64_t>(1, H / 16));
    const int64_t cut = align_up((H + parts - 1) / parts, kRowAlign);
    for (int64_t r0 = 0; r0 < H; r0 += cut) {
      Item it;
      it.h = i32(std::min<int64_t>(cut, H - r0), "item rows");
      it.hpad = i32(align_up(it.h, kRowAlign), "item rows");
      it.out_off = i32(pb[q] + r0, "output row");
      for (int pass = 0; pass < 2; pass++) {
        for (const Cover &e : cov[q]) {
          if (e.kind != pass) continue;
          if (e.kind == 0) {
            EffFull b = eff_full(p, tr, e.k);
            it.segs.push_back({0, e.k, pb[q] + r0 - b.i0, b.n, 0, b.j0});
            it.ncols += b.n;
          } else {
            EffLow b = eff_low(p, tr, e.k);
            if (b.r == 0) continue;
            it.segs.push_back({1, e.k, pb[q] + r0 - b.i0, b.r, 1, op.t_off[e.k]});
            it.ncols += b.r;
          }
        }
      }
      p2.items.push_back(std::move(it));
    }
  }
}

void compute_scales(const Problem &p, bool tr, bool check_finite, OperatorPlan &op) {
  const int64_t nfr = (int64_t)p.fr.size(), nlr = (int64_t)p.lr.size();
  op.scale_fr.assign(nfr, 1.0f);
  op.scale_a.assign(nlr, 1.0f);
  op.scale_b.assign(nlr, 1.0f);
  int64_t bad_fr = -1, bad_lr = -1;
  auto maxabs = [](const View &v, int64_t m, int64_t n, bool &finite) {
    double s = 0.0;
    for (int64_t j = 0; j < n; j++)
      for (int64_t i = 0; i < m; i++) {
        double a = std::fabs(v.at(i, j));
        if (!(a <= 1.0e300)) finite = false;
        s = std::max(s, a);
      }
    return s;
  };
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < nfr; k++) {
    EffFull b = eff_full(p, tr, k);
    bool fin = true;
    double s = maxabs(b.a, b.m, b.n, fin);
    op.scale_fr[k] = (s > 0 && std::isfinite(s)) ? static_cast<float>(s) : 1.0f;
    if (!fin) {
#pragma omp critical
      bad_fr = std::max(bad_fr, k);
    }
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < nlr; k++) {
    EffLow b = eff_low(p, tr, k);
    if (b.r == 0) continue;
    bool fin = true;
    double sa = maxabs(b.A, b.m, b.r, fin);
    double sb = maxabs(b.B, b.r, b.n, fin);
    op.scale_a[k] = (sa > 0 && std::isfinite(sa)) ? static_cast<float>(sa) : 1.0f;
    op.scale_b[k] = (sb > 0 && std::isfinite(sb)) ? static_cast<float>(sb) : 1.0f;
    if (!fin) {
#pragma omp critical
      bad_lr = std::max(bad_lr, k);
    }
  }
  if (check_finite && bad_fr >= 0) fail("non-finite entry in full block " + std::to_string(bad_fr));
  if (check_finite && bad_lr >= 0) fail("non-finite entry in low-rank block " + std::to_string(bad_lr));
  op.t_scale.assign((size_t)std::max<int64_t>(1, op.t_len), 1.0f);
  for (int64_t k = 0; k < nlr; k++) {
    const int64_t r = p.lr[k].r;
    for (int64_t i = 0; i < r; i++) op.t_scale[op.t_off[k] + i] = op.scale_a[k] * op.scale_b[k];
  }
}

void scales_from_maxima(const Problem &p, bool tr, bool check_finite, const double *max_fr, const double *max_a,
                        const double *max_b, const int *nonfinite_fr, const int *nonfinite_lr, OperatorPlan &op) {
  const int64_t nfr = (int64_t)p.fr.size(), nlr = (int64_t)p.lr.size();
  auto scale = [](double s) { return (s > 0 && std::isfinite(s)) ? static_cast<float>(s) : 1.0f; };
  op.scale_fr.assign(nfr, 1.0f);
  op.scale_a.assign(nlr, 1.0f);
  op.scale_b.assign(nlr, 1.0f);
  int64_t bad_fr = -1, bad_lr = -1;
  for (int64_t k = 0; k < nfr; k++) {
    op.scale_fr[k] = scale(max_fr[k]);
    if (nonfinite_fr[k]) bad_fr = k;
  }
  for (int64_t k = 0; k < nlr; k++) {
    if (p.lr[k].r == 0) continue;
    // H^T's factors are B^T and A^T (eff_low): the scales swap
    op.scale_a[k] = scale(tr ? max_b[k] : max_a[k]);
    op.scale_b[k] = scale(tr ? max_a[k] : max_b[k]);
    if (nonfinite_lr[k]) bad_lr = k;
  }
  if (check_finite && bad_fr >= 0) fail("non-finite entry in full block " + std::to_string(bad_fr));
  if (check_finite && bad_lr >= 0) fail("non-finite entry in low-rank block " + std::to_string(bad_lr));
  op.t_scale.assign((size_t)std::max<int64_t>(1, op.t_len), 1.0f);
  for (int64_t k = 0; k < nlr; k++) {
    const int64_t r = p.lr[k].r;
    for (int64_t i = 0; i < r; i++) op.t_scale[op.t_off[k] + i] = op.scale_a[k] * op.scale_b[k];
  }
}

namespace {

// Scale of a G2 run (BF16 only): a full block's scale, or for the t values of
// a low-rank block the product of its two factor scales (phase 1 writes t
// unscaled; the gather applies the product, one FP32 rounding either way).
float seg_scale(const OperatorPlan &op, const Segment &s, int prec) {
  if (prec != 2) return 1.0f;
  if (s.kind == 0) return op.scale_fr[s.block];
  if (s.kind == 1) return op.scale_a[s.block] * op.scale_b[s.block];
  return 1.0f;
}

// Chunks of one item for one precision; phase-2 chunks also get their slice of
// the gather array (g_len grows) and the runs that fill it.
void chunk_item(const OperatorPlan &op, const Item &it, int prec, int phase, int chunk_bytes, std::vector<Chunk> &out,
                std::vector<GatherSeg> &gsegs, int64_t &g_len) {
  const int es = esize_of(prec);
  const bool tiled = prec == 2;
  int64_t cap;
  if (tiled)
    cap = std::max<int64_t>(8, std::min<int64_t>(kMaxCols, (chunk_bytes / (8 * int64_t(it.hpad) * es)) * 8));
  else
    cap = std::max<int64_t>(1, std::min<int64_t>(kMaxCols, chunk_bytes / (int64_t(it.hpad) * es)));
  std::vector<int64_t> seg_start(it.segs.size() + 1, 0);
  for (size_t s = 0; s < it.segs.size(); s++) seg_start[s + 1] = seg_start[s] + it.segs[s].ncols;
  int64_t c0 = 0;
  size_t s_at = 0;  // first segment that may overlap column c0
  do {
    const int64_t take = std::min<int64_t>(cap, it.ncols - c0);
    Chunk ch;
    std::memset(&ch, 0, sizeof ch);
    ch.data_off = it.off[prec] + (tiled ? (c0 / 8) * 8 * int64_t(it.hpad) : c0 * int64_t(it.hpad));
    ch.ncols = i32(take, "chunk columns");
    ch.hpad = it.hpad;
    ch.rows = it.h;
    ch.out_off = it.out_off;
    if (phase == 0) {
      ch.g_off = it.segs.empty() ? 0 : i32(it.segs[0].src_off + c0, "vector offset");
    } else {
      const int64_t g = (g_len + 3) / 4 * 4;  // 16-byte aligned slice in FP32, 32 in FP64
      if (g + take > INT32_MAX) throw std::runtime_error("gather array above 2^31 entries");
      ch.g_off = i32(g, "G2 offset");
      g_len = g + take;
      while (s_at < it.segs.size() && seg_start[s_at + 1] <= c0) s_at++;
      for (size_t s = s_at; s < it.segs.size() && seg_start[s] < c0 + take; s++) {
        const int64_t a = std::max<int64_t>(c0, seg_start[s]), b = std::min<int64_t>(c0 + take, seg_start[s + 1]);
        if (b <= a) continue;
        const Segment &sg = it.segs[s];
        GatherSeg gs;
        gs.dst = i32(g + (a - c0), "G2 offset");
        gs.src_off = i32(sg.src_off + (a - seg_start[s]), "gather source");
        gs.cols_src = u31(b - a, "gather run") | (sg.src ? 0x80000000u : 0u);
        gs.scale = seg_scale(op, sg, prec);
        gsegs.push_back(gs);
      }
    }
    if (out.empty()) ch.flags |= kFirst;
    c0 += take;
    if (c0 >= it.ncols) ch.flags |= kLast;
    out.push_back(ch);
  } while (c0 < it.ncols);
}

}  // namespace

void build_chunks(const Problem &p, bool tr, int prec, int grid, OperatorPlan &op) {
  (void)tr;
  (void)grid;
  const int es = esize_of(prec);
  for (int phase = 0; phase < 2; phase++) {
    PhasePlan &ph = op.ph[phase];
    ChunkPlan &cp = ph.cp[prec];
    // data layout of this precision
    int64_t off = 0;
    for (Item &it : ph.items) {
      it.off[prec] = off;
      off = align_up(off + item_elems(prec, it.hpad, it.ncols), kItemAlign);
    }
    ph.n_elems[prec] = off + kItemAlign;  // slack so 16-byte rounded copies stay inside
    std::vector<std::vector<Chunk>> per_item(ph.items.size());
    cp.gsegs.clear();
    cp.g_len = 0;
    for (size_t q = 0; q < ph.items.size(); q++)
      chunk_item(op, ph.items[q], prec, phase, p.tune.chunk_bytes, per_item[q], cp.gsegs, cp.g_len);
    // Longest first: the CTAs take items from a queue in this order (greedy
    // list scheduling; each CTA takes the next item when its producer is
    // done with the previous one).  Cost is the bytes streamed plus a fixed
    // per-chunk overhead (descriptor, barrier round trip) expressed in bytes.
    const int64_t n = (int64_t)ph.items.size();
    std::vector<int64_t> cost(n);
    for (int64_t q = 0; q < n; q++)
      cost[q] = item_elems(prec, ph.items[q].hpad, ph.items[q].ncols) * es + 1024 * (int64_t)per_item[q].size();
    std::vector<int64_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    // Queue units: runs of consecutive items, closed once their cost
    // reaches unit_bytes (a large item is a unit by itself).  The kernel
    // walks a unit's chunks as one range; item boundaries stay in the chunk
    // flags, so results do not depend on the grouping.
    cp.chunks.clear();
    cp.item_ptr.assign(1, 0);
    int64_t unit_cost = 0;
    for (size_t k = 0; k < order.size(); k++) {
      const int64_t q = order[k];
      cp.chunks.insert(cp.chunks.end(), per_item[q].begin(), per_item[q].end());
      if (cp.chunks.size() > (size_t)INT32_MAX) fail("too many chunks");
      unit_cost += cost[q];
      if (unit_cost >= p.tune.unit_bytes || k + 1 == order.size()) {
        cp.item_ptr.push_back(i32((int64_t)cp.chunks.size(), "chunk count"));
        unit_cost = 0;
      }
    }
  }
}

namespace {

// One column run of an item: rows [r0, r0 + n) of item column c from
// src[i * stride], converted to the precision's storage (FP32: rounded; BF16:
// times inv, rounded to FP32 then BF16) at the item_index positions.
template <int PREC>
inline void put_run(void *dst, int64_t e0, int64_t hpad, int64_t r0, int64_t c, const double *src, int64_t stride,
                    int64_t n, double inv) {
  if constexpr (PREC == 0) {
    double *d = static_cast<double *>(dst) + e0 + c * hpad + r0;
    if (stride == 1)
      std::memcpy(d, src, sizeof(double) * (size_t)n);
    else
      for (int64_t i = 0; i < n; i++) d[i] = src[i * stride];
  } else if constexpr (PREC == 1) {
    float *d = static_cast<float *>(dst) + e0 + c * hpad + r0;
    for (int64_t i = 0; i < n; i++) d[i] = static_cast<float>(src[i * stride]);
  } else {
    uint16_t *d = static_cast<uint16_t *>(dst) + e0 + (c >> 3) * (8 * hpad) + (c & 7) * 8;
    for (int64_t i = 0; i < n; i++) {
      const int64_t r = r0 + i;
      d[(r >> 3) * 64 + (r & 7)] = to_bf16(static_cast<float>(src[i * stride] * inv));
    }
  }
}

// Column c of a view from row r0 on, as (pointer, stride).
inline const double *view_column(const View &v, int64_t r0, int64_t c, int64_t &stride) {
  stride = v.trans ? v.ld : 1;
  return v.trans ? v.p + r0 * v.ld + c : v.p + r0 + c * v.ld;
}

template <int PREC>
void fill_items_t(const Problem &p, bool tr, const OperatorPlan &op, int phase, int64_t i_begin, int64_t i_end,
                  int64_t base, void *dst) {
  const PhasePlan &ph = op.ph[phase];
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t q = i_begin; q < i_end; q++) {
    const Item &it = ph.items[q];
    const int64_t e0 = it.off[PREC] - base;
    int64_t stride;
    if (phase == 0) {  // stacked B rows, one segment of columns
      int64_t row = 0;
      for (const RowPiece &pc : it.pieces) {
        const View B = eff_low(p, tr, pc.block).B;
        const double inv = PREC == 2 ? 1.0 / op.scale_b[pc.block] : 1.0;
        for (int64_t c = 0; c < it.ncols; c++) {
          const double *src = view_column(B, pc.r0, c, stride);
          put_run<PREC>(dst, e0, it.hpad, row, c, src, stride, pc.n, inv);
        }
        row += pc.n;
      }
      continue;
    }
    int64_t col = 0;
    for (const Segment &sg : it.segs) {
      View v;
      double inv = 1.0;
      if (sg.kind == 0) {
        v = eff_full(p, tr, sg.block).a;
        if (PREC == 2) inv = 1.0 / op.scale_fr[sg.block];
      } else {
        v = eff_low(p, tr, sg.block).A;
        if (PREC == 2) inv = 1.0 / op.scale_a[sg.block];
      }
      for (int64_t c = 0; c < sg.ncols; c++) {
        const double *src = view_column(v, sg.row0, c, stride);
        put_run<PREC>(dst, e0, it.hpad, 0, col + c, src, stride, it.h, inv);
      }
      col += sg.ncols;
    }
  }
}

}  // namespace

void fill_items(const Problem &p, bool tr, const OperatorPlan &op, int phase, int prec, int64_t i_begin,
                int64_t i_end, int64_t base, void *dst) {
  if (prec == 0)
    fill_items_t<0>(p, tr, op, phase, i_begin, i_end, base, dst);
  else if (prec == 1)
    fill_items_t<1>(p, tr, op, phase, i_begin, i_end, base, dst);
  else
    fill_items_t<2>(p, tr, op, phase, i_begin, i_end, base, dst);
}

void build_pack_runs(const Problem &p, bool tr, const OperatorPlan &op, int phase, int prec, const double *fr_base,
                     int64_t fr_len, const double *lr_base, int64_t lr_len, std::vector<PackRun> &out) {
  const PhasePlan &ph = op.ph[phase];
  out.clear();
  auto locate = [&](const View &v, int64_t rows, int64_t cols, PackRun &r) {
    // every element of the view the run reads must lie in its array
    const int64_t span = v.trans ? (rows - 1) * v.ld + cols : (cols - 1) * v.ld + rows;
    if (v.p >= fr_base && v.p + span <= fr_base + fr_len) {
      r.array = 0;
      r.src_off = v.p - fr_base;
    } else if (v.p >= lr_base && v.p + span <= lr_base + lr_len) {
      r.array = 1;
      r.src_off = v.p - lr_base;
    } else {
      throw std::invalid_argument("build_pack_runs: a block view lies outside the flat block arrays");
    }
    r.ld = v.ld;
    r.trans = v.trans ? 1 : 0;
  };
  for (const Item &it : ph.items) {
    PackRun r;
    std::memset(&r, 0, sizeof r);
    r.item_off = it.off[prec];
    r.hpad = it.hpad;
    if (phase == 0) {
      int64_t row = 0;
      for (const RowPiece &pc : it.pieces) {
        const EffLow e = eff_low(p, tr, pc.block);
        locate(e.B, e.r, e.n, r);
        r.inv = prec == 2 ? 1.0 / op.scale_b[pc.block] : 1.0;
        r.dst_r0 = i32(row, "item row");
        r.dst_c0 = 0;
        r.src_r0 = i32(pc.r0, "factor row");
        r.src_c0 = 0;
        r.n = i32(pc.n, "rows");
        r.ncols = i32(it.ncols, "columns");
        out.push_back(r);
        row += pc.n;
      }
      continue;
    }
    int64_t col = 0;
    for (const Segment &sg : it.segs) {
      if (sg.kind == 0) {
        const EffFull e = eff_full(p, tr, sg.block);
        locate(e.a, e.m, e.n, r);
        r.inv = prec == 2 ? 1.0 / op.scale_fr[sg.block] : 1.0;
      } else {
        const EffLow e = eff_low(p, tr, sg.block);
        locate(e.A, e.m, e.r, r);
        r.inv = prec == 2 ? 1.0 / op.scale_a[sg.block] : 1.0;
      }
      r.dst_r0 = 0;
      r.dst_c0 = i32(col, "item column");
      r.src_r0 = i32(sg.row0, "block row");
      r.src_c0 = 0;
      r.n = it.h;
      r.ncols = i32(sg.ncols, "columns");
      out.push_back(r);
      col += sg.ncols;
    }
  }
}

// ---------------------------------------------------------------------------- matmat plan

namespace {

// Chunks of one matmat item: at most kMmMaxCols columns and kMmStageBytes of
// block data + operand rows, multiples of 16 columns, at most kMmMaxRuns runs.
void mm_chunk_item(const MmItem &it, std::vector<MmChunk> &out) {
  const int64_t per_col = 2 * int64_t(it.hpad) + 2 * int64_t(kMmRhs);
  const int64_t cap = std::max<int64_t>(16, std::min<int64_t>(kMmMaxCols, (kMmStageBytes / per_col) / 16 * 16));
  std::vector<int64_t> seg_start(it.segs.size() + 1, 0);
  for (size_t s = 0; s < it.segs.size(); s++) seg_start[s + 1] = seg_start[s] + it.segs[s].ncols;
  int64_t c0 = 0;
  size_t s_at = 0;
  while (c0 < it.ncols) {
    while (s_at < it.segs.size() && seg_start[s_at + 1] <= c0) s_at++;
    MmChunk ch;
    std::memset(&ch, 0, sizeof ch);
    // runs until the column cap or the run cap; the chunk must end on a
    // multiple of 16 columns, so a fourth run may be cut short
    int64_t end = std::min<int64_t>(c0 + cap, it.ncols);
    int nr = 0;
    for (size_t s = s_at; s < it.segs.size() && seg_start[s] < end; s++) {
      if (nr == kMmMaxRuns) {
        end = seg_start[s];
        break;
      }
      nr++;
    }
    end = c0 + (end - c0) / 16 * 16;
    if (end <= c0) end = std::min<int64_t>(c0 + 16, it.ncols);  // segments of 8: the run cap bends to fit 16 columns
    nr = 0;
    for (size_t s = s_at; s < it.segs.size() && seg_start[s] < end; s++) {
      const int64_t a = std::max<int64_t>(c0, seg_start[s]), b = std::min<int64_t>(end, seg_start[s + 1]);
      if (b <= a) continue;
      if (nr == kMmMaxRuns) throw std::runtime_error("matmat chunk needs more than the run cap");
      const MmSeg &sg = it.segs[s];
      ch.run[nr].src = u31(sg.src_row + (a - seg_start[s]), "operand row") | (sg.src ? 0x80000000u : 0u);
      ch.run[nr].rows = u31(b - a, "operand rows");
      nr++;
    }
    ch.data_off = it.off + (c0 / 8) * 8 * int64_t(it.hpad);
    ch.kc = i32(end - c0, "chunk columns");
    ch.hpad = it.hpad;
    ch.rows = it.h;
    ch.out_off = it.out_off;
    ch.flags = static_cast<uint32_t>(nr) << 8;
    if (c0 == 0) ch.flags |= kFirst;
    if (end >= it.ncols) ch.flags |= kLast;
    out.push_back(ch);
    c0 = end;
  }
}

}  // namespace

void build_mm_plan(const Problem &p, bool tr, int grid, const OperatorPlan &op, MmPlan &mm) {
  mm = MmPlan{};
  mm.n_in = op.n_in;
  mm.n_out = op.n_out;
  const size_t nlr = p.lr.size();
  grid = std::max(1, grid);
  // stacks per column cluster (the matvec's phase-1 grouping), T8 numbering
  std::map<std::pair<int64_t, int64_t>, std::vector<int64_t>> stacks;
  for (size_t k = 0; k < nlr; k++) {
    EffLow b = eff_low(p, tr, k);
    if (b.r > 0) stacks[{b.j0, b.n}].push_back((int64_t)k);
  }
  mm.t8_off.assign(nlr, 0);
  int64_t t8 = 0;
  for (auto &kv : stacks) {
    MmStack st{kv.first.first, kv.first.second, kv.second, t8};
    for (int64_t k : kv.second) {
      mm.t8_off[k] = t8;
      t8 += align_up(eff_low(p, tr, k).r, 8);
    }
    mm.stacks.push_back(std::move(st));
  }
  mm.t8_len = t8;
  if (t8 + kMmPadRows > INT32_MAX) fail("padded sum of ranks above 2^31");
  // phase 1: each stack's rows cut into items of at most kHMax rows
  int64_t e1 = 0;
  std::vector<int64_t> wcols(mm.stacks.size()), rows8(mm.stacks.size());
  for (size_t s = 0; s < mm.stacks.size(); s++) {
    const MmStack &st = mm.stacks[s];
    const int64_t j0a = st.j0 / 8 * 8;
    wcols[s] = std::max<int64_t>(kMmMinCols, align_up(st.j0 + st.n - j0a, 16));
    int64_t R8 = 0;
    for (int64_t k : st.blocks) R8 += align_up(eff_low(p, tr, k).r, 8);
    rows8[s] = R8;
    e1 += R8 * wcols[s];
  }
  const int64_t cap1 = std::max<int64_t>(1, e1 / grid / std::max(1, p.tune.mm_items_per_cta));
  MmPhase &p1 = mm.ph[0];
  for (size_t s = 0; s < mm.stacks.size(); s++) {
    const MmStack &st = mm.stacks[s];
    const int64_t W = wcols[s], R8 = rows8[s];
    const int64_t rmax = std::min<int64_t>(kMmHMax, std::max<int64_t>(16, (cap1 / W) / 16 * 16));
    const int64_t nit = (R8 + rmax - 1) / rmax;
    const int64_t cut = align_up((R8 + nit - 1) / nit, 8);
    for (int64_t r0 = 0; r0 < R8; r0 += cut) {
      MmItem it;
      it.h = i32(std::min<int64_t>(cut, R8 - r0), "item rows");
      it.hpad = it.h;
      it.out_off = i32(st.t8_base + r0, "T8 offset");
      it.ncols = W;
      it.stack = (int64_t)s;
      it.srow0 = r0;
      const int64_t j0a = st.j0 / 8 * 8;
      it.segs.push_back({2, -1, 0, st.j0 - j0a, st.n, W, 0, j0a});
      p1.items.push_back(std::move(it));
    }
  }
  // phase 2: the matvec's row-panel items on widened windows, cut into parts
  // of at most kMmHMax rows
  MmPhase &p2 = mm.ph[1];
  auto window = [&](const Segment &sg, int64_t r0) {
    MmSeg m{};
    m.kind = sg.kind;
    m.block = sg.block;
    m.row0 = sg.row0 + r0;
    if (sg.kind == 0) {
      m.src = 0;
      m.src_row = sg.src_off / 8 * 8;
      m.lead = sg.src_off - m.src_row;
    } else {
      m.src = 1;
      m.src_row = mm.t8_off[sg.block];
      m.lead = 0;
    }
    m.width = sg.ncols;  // the block's columns, or its rank
    m.ncols = align_up(m.lead + m.width, 8);
    return m;
  };
  for (const Item &src : op.ph[1].items) {
    const int64_t parts = (src.hpad + kMmHMax - 1) / kMmHMax;
    const int64_t cut = align_up((src.h + parts - 1) / parts, 8);
    for (int64_t r0 = 0; r0 < src.h; r0 += cut) {
      MmItem it;
      it.h = i32(std::min<int64_t>(cut, src.h - r0), "item rows");
      it.hpad = i32(align_up(it.h, 8), "item rows");
      it.out_off = i32(src.out_off + r0, "output row");
      for (const Segment &sg : src.segs) {
        it.segs.push_back(window(sg, r0));
        it.ncols += it.segs.back().ncols;
      }
      if (it.segs.empty()) {
        // every block of the panel has rank 0: one window of zero block
        // columns over T8's zeroed padding rows, so the rows are written (as 0)
        MmSeg z{};
        z.kind = 1;
        z.block = -1;
        z.src = 1;
        z.src_row = mm.t8_len;
        it.segs.push_back(z);
      }
      // a multiple of 16 columns, at least kMmMinCols: more tile rows of the
      // last operand window (zero columns)
      const int64_t want = std::max<int64_t>(kMmMinCols, align_up(it.ncols, 16));
      it.segs.back().ncols += want - it.ncols;
      it.ncols = want;
      p2.items.push_back(std::move(it));
    }
  }
  // data offsets, chunks, items longest first (cost: block bytes + operand bytes + a per-chunk overhead)
  for (int phase = 0; phase < 2; phase++) {
    MmPhase &ph = mm.ph[phase];
    int64_t off = 0;
    for (MmItem &it : ph.items) {
      it.off = off;
      off = align_up(off + it.ncols * int64_t(it.hpad), kItemAlign);
    }
    ph.n_elems = off + kItemAlign;
    std::vector<std::vector<MmChunk>> per_item(ph.items.size());
    std::vector<int64_t> cost(ph.items.size(), 0);
    for (size_t q = 0; q < ph.items.size(); q++) {
      mm_chunk_item(ph.items[q], per_item[q]);
      for (const MmChunk &c : per_item[q]) cost[q] += int64_t(c.kc) * (2 * c.hpad + 2 * kMmRhs) + 1024;
    }
    std::vector<int64_t> order(ph.items.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    ph.chunks.clear();
    ph.item_ptr.assign(1, 0);
    for (int64_t q : order) {
      ph.chunks.insert(ph.chunks.end(), per_item[q].begin(), per_item[q].end());
      if (ph.chunks.size() > (size_t)INT32_MAX) fail("too many matmat chunks");
      ph.item_ptr.push_back(i32((int64_t)ph.chunks.size(), "chunk count"));
    }
  }
}

void fill_mm_items(const Problem &p, bool tr, const MmPlan &mm, int phase, int64_t i_begin, int64_t i_end,
                   int64_t base, uint16_t *dst) {
  const MmPhase &ph = mm.ph[phase];
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t q = i_begin; q < i_end; q++) {
    const MmItem &it = ph.items[q];
    uint16_t *d = dst + (it.off - base);
    if (phase == 0) {
      // stack rows [srow0, srow0 + h): block rows, then zero rows up to the
      // block's padded rank; columns: the window [j0a, j0a + ncols)
      const MmStack &st = mm.stacks[it.stack];
      const MmSeg &sg = it.segs[0];
      int64_t sb = 0;  // stack row of the current block's first row
      for (int64_t k : st.blocks) {
        const EffLow b = eff_low(p, tr, k);
        const int64_t r8 = align_up(b.r, 8);
        const int64_t lo = std::max<int64_t>(sb, it.srow0), hi = std::min<int64_t>(sb + b.r, it.srow0 + it.h);
        for (int64_t s = lo; s < hi; s++)
          for (int64_t c = 0; c < sg.width; c++)
            d[item_index(2, it.hpad, s - it.srow0, sg.lead + c)] = to_bf16(static_cast<float>(b.B.at(s - sb, c)));
        sb += r8;
        if (sb >= it.srow0 + it.h) break;
      }
      continue;
    }
    int64_t col = 0;
    for (const MmSeg &s : it.segs) {
      if (s.width == 0) {  // a panel of rank-0 blocks only: zero columns
        col += s.ncols;
        continue;
      }
      const View v = s.kind == 0 ? eff_full(p, tr, s.block).a : eff_low(p, tr, s.block).A;
      for (int64_t c = 0; c < s.width; c++)
        for (int64_t i = 0; i < it.h; i++)
          d[item_index(2, it.hpad, i, col + s.lead + c)] = to_bf16(static_cast<float>(v.at(s.row0 + i, c)));
      col += s.ncols;
    }
  }
}

}  // namespace bw
